/*
 * qv_oracle.c -- CPU restatement of Qvort's velocity-and-timestep path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * qvort_b200/csrc: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs may load it.  The product library never links or calls it.
 *
 * It restates, in plain C with FP64 arithmetic and no FMA contraction
 * (build with -O2 -ffp-contract=off -fno-fast-math), the reference Fortran
 * routines below.  gfortran -O2 on x86-64 evaluates same-precedence
 * operators left to right, expands x**2, x**3 and x**5 into multiplications
 * and does not reassociate floating-point sums; the C below writes every
 * expression in that same order.  File:line citations are to the reference
 * project (abag/qvort, src/).
 *
 * Parity status: the reference ships no tests, fixtures or golden vectors for
 * this path and no Fortran compiler is available to run it, so this oracle is
 * "parity unpinned" against reference outputs.  It is pinned instead against
 * analytic known answers the reference itself prints (ring self-induced
 * velocity, src/initial_loop.f90:17-19) and against hand-checked small cases.
 *
 * Conventions: n slots; positions and vectors are interleaved x[3*i+c];
 * infront/behind hold 1-based indices with 0 marking an empty slot
 * (src/cdata.f90:20-39, src/timestep.f90:43).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define QO_PI 3.14159265358979324 /* src/cdata.f90:176 */
#define QO_EPS 2.220446049250313e-16 /* epsilon(0.) with -fdefault-real-8 */

typedef struct {
  double quant_circ, corea, box_size, delta, dt, tree_theta;
  int boundary;   /* 0 open, 1 periodic, 2 openx (periodic y,z), 3 openxy (periodic z) */
  int velocity;   /* 0 Off, 1 LIA, 2 BS, 3 Tree */
  int deriv_order;/* 2 or 4 */
  int tree_extra_correction;
  int fixed_lia_beta;
} qo_params;

/* ---------------------------------------------------------------- helpers */
static inline double sq(double a) { return a * a; }

/* dist_gen, src/derivatives.f90:79-86 */
static inline double dist_gen(const double *a, const double *b) {
  return sqrt(sq(a[0] - b[0]) + sq(a[1] - b[1]) + sq(a[2] - b[2]));
}
/* dist_gen_sq, src/general.f90:58-65 */
static inline double dist_gen_sq(const double *a, const double *b) {
  return sq(a[0] - b[0]) + sq(a[1] - b[1]) + sq(a[2] - b[2]);
}
/* cross_product, src/general.f90:142-149 */
static inline void cross(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
static inline double dot3(const double *a, const double *b) {
  double s = a[0] * b[0];
  s = s + a[1] * b[1];
  s = s + a[2] * b[2];
  return s;
}

/* eps(3,3,3), src/cdata.f90:183-189 (Levi-Civita, eps(1,2,3)=1) */
static double levi(int m, int k, int l) {
  if (m == k || k == l || m == l) return 0.0;
  if ((m == 0 && k == 1 && l == 2) || (m == 1 && k == 2 && l == 0) ||
      (m == 2 && k == 0 && l == 1))
    return 1.0;
  return -1.0;
}

/* ------------------------------------------------------------ ghost points */
/* get_ghost_p, src/periodic.f90:23-165 (mirror branch out of scope) */
static void unwrap(const qo_params *p, const double *xi, double *g, int axis) {
  double h = p->box_size / 2.;
  if ((xi[axis] - g[axis]) > h)
    g[axis] = g[axis] + p->box_size;
  else if ((xi[axis] - g[axis]) < (-h))
    g[axis] = g[axis] - p->box_size;
}

void qo_ghosts(const qo_params *p, int n, const double *x, const int *infront,
               const int *behind, double *gi, double *gb, double *gii,
               double *gbb) {
  for (int i = 0; i < n; i++) {
    if (infront[i] == 0) continue;
    int a = infront[i] - 1, b = behind[i] - 1;
    int aa = infront[a] - 1, bb = behind[b] - 1;
    double *G[4] = {gi + 3 * i, gb + 3 * i, gii + 3 * i, gbb + 3 * i};
    int src[4] = {a, b, aa, bb};
    for (int k = 0; k < 4; k++)
      for (int c = 0; c < 3; c++) G[k][c] = x[3 * src[k] + c];
    int lo = 3; /* no periodic axes */
    if (p->boundary == 1) lo = 0;
    else if (p->boundary == 2) lo = 1;
    else if (p->boundary == 3) lo = 2;
    /* the reference handles axis x for all four ghosts, then y, then z */
    for (int axis = lo; axis < 3; axis++)
      for (int k = 0; k < 4; k++) unwrap(p, x + 3 * i, G[k], axis);
  }
}

/* enforce_periodic, src/periodic.f90:188-214 (and the yz / z variants) */
void qo_enforce_periodic(const qo_params *p, int n, double *x, const int *infront) {
  int lo = 3;
  if (p->boundary == 1) lo = 0;
  else if (p->boundary == 2) lo = 1;
  else if (p->boundary == 3) lo = 2;
  double h = p->box_size / 2.;
  for (int i = 0; i < n; i++) {
    if (infront[i] == 0) continue;
    for (int c = lo; c < 3; c++) {
      if (x[3 * i + c] > h)
        x[3 * i + c] = x[3 * i + c] - p->box_size;
      else if (x[3 * i + c] < (-h))
        x[3 * i + c] = x[3 * i + c] + p->box_size;
    }
  }
}

/* ------------------------------------------------------------ derivatives */
/* get_deriv_1, src/derivatives.f90:11-39 */
static void deriv1(const qo_params *p, const double *x, const double *gi,
                   const double *gb, const double *gii, const double *gbb,
                   double *s) {
  double disti = dist_gen(x, gi), distb = dist_gen(x, gb);
  if (p->deriv_order != 4) {
    for (int c = 0; c < 3; c++)
      s[c] = distb * gi[c] + (disti - distb) * x[c] - disti * gb[c];
    for (int c = 0; c < 3; c++) s[c] = s[c] / (2. * distb * disti);
  } else {
    double dii = dist_gen(gii, gi), dbb = dist_gen(gbb, gb);
    double A = distb * sq(disti) + distb * disti * dii;
    A = A / (dbb * (dbb + distb) * (dbb + distb + disti) * (dbb + distb + disti + dii));
    double B = -dbb * sq(disti) - distb * sq(disti) - dbb * disti * dii - distb * disti * dii;
    B = B / (dbb * distb * (distb + disti) * (distb + disti + dii));
    double D = dbb * distb * disti + sq(distb) * disti + dbb * distb * dii + sq(distb) * dii;
    D = D / (disti * dii * (distb + disti) * (dbb + distb + disti));
    double E = -disti * sq(distb) - dbb * distb * disti;
    E = E / (dii * (disti + dii) * (distb + disti + dii) * (dbb + distb + disti + dii));
    double C = -(A + B + D + E);
    for (int c = 0; c < 3; c++)
      s[c] = A * gbb[c] + B * gb[c] + C * x[c] + D * gi[c] + E * gii[c];
  }
}

/* get_deriv_2, src/derivatives.f90:47-75 */
static void deriv2(const qo_params *p, const double *x, const double *gi,
                   const double *gb, const double *gii, const double *gbb,
                   double *s) {
  double disti = dist_gen(x, gi), distb = dist_gen(x, gb);
  if (p->deriv_order != 4) {
    for (int c = 0; c < 3; c++)
      s[c] = 2. * (gi[c] / (disti * (disti + distb)) - x[c] / (disti * distb) +
                   gb[c] / (distb * (disti + distb)));
  } else {
    double dii = dist_gen(gii, gi), dbb = dist_gen(gbb, gb);
    double A = 2. * (-2. * distb * disti + sq(disti) - distb * dii + disti * dii);
    A = A / (dbb * (dbb + distb) * (dbb + distb + disti) * (dbb + distb + disti + dii));
    double B = 2. * (2. * dbb * disti + 2. * distb * disti - sq(disti) + dbb * dii + distb * dii - disti * dii);
    B = B / (dbb * distb * (distb + disti) * (distb + disti + dii));
    double D = 2. * (-dbb * distb - sq(distb) + dbb * disti + 2. * distb * disti + dbb * dii + 2. * distb * dii);
    D = D / (disti * dii * (distb + disti) * (dbb + distb + disti));
    double E = 2. * (dbb * distb + sq(distb) - dbb * disti - 2. * distb * disti);
    E = E / (dii * (disti + dii) * (distb + disti + dii) * (dbb + distb + disti + dii));
    double C = -(A + B + D + E);
    for (int c = 0; c < 3; c++)
      s[c] = A * gbb[c] + B * gb[c] + C * x[c] + D * gi[c] + E * gii[c];
  }
}

/* ---------------------------------------------------------------- the tree */
typedef struct qo_node {
  double posx, posy, posz, width;
  int pcount;
  struct qo_node *child[8]; /* fbl fbr ftl ftr bbl bbr btl btr; NULL if leaf */
  int *idx;                 /* 0-based indices of the node's points, ascending */
  int nidx;
  double cent[3], circ[3], Cij[3][3];
  int first;          /* 0-based index of parray(1) or -1 */
  int first_infront;  /* parray(1)%infront at build time (1-based) */
  double first_x[3], first_gi[3];
} qo_node;

typedef struct {
  qo_node *root;
  int nnodes, maxdepth, status;
} qo_tree;

static int g_depth_cap = 200;

/* new_tree, src/tree.f90:129-186 */
static qo_node *new_node(double posx, double posy, double posz, double width,
                         const qo_node *parent, const double *x,
                         const double *gi, const int *infront) {
  qo_node *t = (qo_node *)calloc(1, sizeof(qo_node));
  t->posx = posx; t->posy = posy; t->posz = posz; t->width = width;
  t->idx = (int *)malloc(sizeof(int) * (parent->nidx > 0 ? parent->nidx : 1));
  t->first = -1;
  double centx = 0., centy = 0., centz = 0.;
  double circ[3] = {0., 0., 0.};
  double C[3][3] = {{0}};
  int counter = 0;
  for (int q = 0; q < parent->nidx; q++) {
    int i = parent->idx[q];
    if (infront[i] == 0) continue;
    const double *xi = x + 3 * i, *gii = gi + 3 * i;
    if ((xi[0] >= posx) && (xi[0] < (posx + width)) && (xi[1] >= posy) &&
        (xi[1] < (posy + width)) && (xi[2] >= posz) && (xi[2] < (posz + width))) {
      t->idx[counter++] = i;
      centx = centx + xi[0];
      centy = centy + xi[1];
      centz = centz + xi[2];
      for (int c = 0; c < 3; c++) circ[c] = circ[c] + gii[c] - xi[c];
      for (int k = 0; k < 3; k++)
        for (int m = 0; m < 3; m++) C[m][k] = C[m][k] + xi[m] * (gii[k] - xi[k]);
    }
  }
  t->nidx = counter;
  t->pcount = counter;
  t->cent[0] = t->cent[1] = t->cent[2] = 0.;
  if (counter != 0) {
    centx = centx / counter;
    centy = centy / counter;
    centz = centz / counter;
    t->cent[0] = centx; t->cent[1] = centy; t->cent[2] = centz;
    for (int i = 0; i < 3; i++)
      for (int k = 0; k < 3; k++) C[i][k] = C[i][k] - t->cent[i] * circ[k];
    int f = t->idx[0];
    t->first = f;
    t->first_infront = infront[f];
    for (int c = 0; c < 3; c++) { t->first_x[c] = x[3 * f + c]; t->first_gi[c] = gi[3 * f + c]; }
  }
  memcpy(t->circ, circ, sizeof circ);
  memcpy(t->Cij, C, sizeof C);
  return t;
}

/* build_tree, src/tree.f90:85-125 */
static void build_rec(qo_tree *T, qo_node *t, int depth, const double *x,
                      const double *gi, const int *infront) {
  T->nnodes++;
  if (depth > T->maxdepth) T->maxdepth = depth;
  if (t->pcount > 1) {
    if (depth >= g_depth_cap) { T->status = -2; return; }
    double w = t->width / 2.;
    double px = t->posx, py = t->posy, pz = t->posz;
    double pxw = t->posx + (t->width / 2), pyw = t->posy + (t->width / 2),
           pzw = t->posz + (t->width / 2);
    t->child[0] = new_node(px, py, pz, w, t, x, gi, infront);    /* fbl */
    t->child[1] = new_node(pxw, py, pz, w, t, x, gi, infront);   /* fbr */
    t->child[2] = new_node(px, py, pzw, w, t, x, gi, infront);   /* ftl */
    t->child[3] = new_node(pxw, py, pzw, w, t, x, gi, infront);  /* ftr */
    t->child[4] = new_node(px, pyw, pz, w, t, x, gi, infront);   /* bbl */
    t->child[5] = new_node(pxw, pyw, pz, w, t, x, gi, infront);  /* bbr */
    t->child[6] = new_node(px, pyw, pzw, w, t, x, gi, infront);  /* btl */
    t->child[7] = new_node(pxw, pyw, pzw, w, t, x, gi, infront); /* btr */
    for (int k = 0; k < 8; k++) build_rec(T, t->child[k], depth + 1, x, gi, infront);
  }
}

/* construct_tree, src/tree.f90:44-80 */
qo_tree *qo_tree_build(const qo_params *p, int n, const double *x,
                       const double *gi, const int *infront) {
  qo_tree *T = (qo_tree *)calloc(1, sizeof(qo_tree));
  qo_node *r = (qo_node *)calloc(1, sizeof(qo_node));
  r->posx = -p->box_size / 2.;
  r->posy = -p->box_size / 2.;
  r->posz = -p->box_size / 2.;
  r->width = p->box_size;
  r->pcount = n;
  r->nidx = n;
  r->idx = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++) r->idx[i] = i;
  double s[3] = {0., 0., 0.};
  int cnt = 0;
  for (int i = 0; i < n; i++)
    if (infront[i] > 0) cnt++;
  for (int c = 0; c < 3; c++)
    for (int i = 0; i < n; i++)
      if (infront[i] > 0) s[c] = s[c] + x[3 * i + c];
  for (int c = 0; c < 3; c++) r->cent[c] = s[c] / cnt;
  r->first = n > 0 ? 0 : -1;
  if (n > 0) {
    r->first_infront = infront[0];
    for (int c = 0; c < 3; c++) { r->first_x[c] = x[c]; r->first_gi[c] = gi[c]; }
  }
  T->root = r;
  build_rec(T, r, 0, x, gi, infront);
  return T;
}

static void free_rec(qo_node *t) {
  for (int k = 0; k < 8; k++)
    if (t->child[k]) free_rec(t->child[k]);
  free(t->idx);
  free(t);
}
void qo_tree_free(qo_tree *T) {
  if (!T) return;
  if (T->root) free_rec(T->root);
  free(T);
}
int qo_tree_status(const qo_tree *T) { return T->status; }
int qo_tree_maxdepth(const qo_tree *T) { return T->maxdepth; }

/* Count of non-empty nodes (the root always counts). */
static int count_nonempty(const qo_node *t, int is_root) {
  int c = (is_root || t->pcount > 0) ? 1 : 0;
  for (int k = 0; k < 8; k++)
    if (t->child[k]) c += count_nonempty(t->child[k], 0);
  return c;
}
int qo_tree_count(const qo_tree *T) { return count_nonempty(T->root, 1); }

/*
 * Export the non-empty nodes in breadth-first order, children in the fixed
 * fbl..btr order.  This is the canonical order the GPU builder also emits.
 * Per node: parent (BFS index, -1 for the root), child digit, depth, corner,
 * width, pcount, cent, circ, Cij (row-major C[i][k]), first point (0-based).
 */
int qo_tree_export(const qo_tree *T, int cap, int *parent, int *digit, int *depth,
                   double *pos, double *width, int *pcount, double *cent,
                   double *circ, double *Cij, int *first) {
  int total = qo_tree_count(T);
  if (total > cap) return -total;
  const qo_node **q = (const qo_node **)malloc(sizeof(void *) * total);
  int *qp = (int *)malloc(sizeof(int) * total), *qd = (int *)malloc(sizeof(int) * total),
      *qdep = (int *)malloc(sizeof(int) * total);
  int head = 0, tail = 0;
  q[tail] = T->root; qp[tail] = -1; qd[tail] = -1; qdep[tail] = 0; tail++;
  while (head < tail) {
    const qo_node *t = q[head];
    int me = head++;
    parent[me] = qp[me]; digit[me] = qd[me]; depth[me] = qdep[me];
    pos[3 * me] = t->posx; pos[3 * me + 1] = t->posy; pos[3 * me + 2] = t->posz;
    width[me] = t->width; pcount[me] = t->pcount; first[me] = t->first;
    for (int c = 0; c < 3; c++) { cent[3 * me + c] = t->cent[c]; circ[3 * me + c] = t->circ[c]; }
    for (int i = 0; i < 3; i++)
      for (int k = 0; k < 3; k++) Cij[9 * me + 3 * i + k] = t->Cij[i][k];
    for (int k = 0; k < 8; k++) {
      const qo_node *c = t->child[k];
      if (c && c->pcount > 0) {
        q[tail] = c; qp[tail] = me; qd[tail] = k; qdep[tail] = qdep[me] + 1; tail++;
      }
    }
  }
  free(q); free(qp); free(qd); free(qdep);
  return total;
}

/* ---------------------------------------------------------- tree_walk */
typedef struct {
  const qo_params *p;
  int i;
  const double *xi;
  const int *infront, *behind;
  long long evals;
  int status;
} walk_ctx;

/* tree_walk, src/tree.f90:336-421 */
static void tree_walk(walk_ctx *W, const qo_node *t, const double *shift, double *u) {
  const qo_params *p = W->p;
  int i = W->i;
  if (W->infront[i] == 0) return;
  if (t->pcount == 0) return;
  const double *xi = W->xi;
  double dist = sqrt(sq(xi[0] - (t->cent[0] + shift[0])) + sq(xi[1] - (t->cent[1] + shift[1])) +
                     sq(xi[2] - (t->cent[2] + shift[2])));
  double theta;
  if (p->tree_extra_correction) {
    double geo = sqrt(sq(t->cent[0] - (t->posx + t->width / 2.)) +
                      sq(t->cent[1] - (t->posy + t->width / 2.)) +
                      sq(t->cent[2] - (t->posz + t->width / 2.)));
    if (dist - geo > 0.)
      theta = t->width / (dist - geo);
    else
      theta = t->width / dist;
  } else {
    theta = t->width / dist;
  }
  if (t->pcount == 1) {
    int j = W->behind[t->first_infront - 1]; /* f(parray(1)%infront)%behind, 1-based */
    if (j == i + 1) return;
    if (j == W->behind[i]) return;
    if (j == W->infront[i]) return;
    if (dist < QO_EPS) { W->status = -1; return; }
    double R1[3], R2[3], cr[3];
    for (int c = 0; c < 3; c++) {
      R1[c] = t->first_x[c] + shift[c] - xi[c];
      R2[c] = t->first_gi[c] + shift[c] - xi[c];
    }
    double a = sqrt(dot3(R1, R1));
    double b = sqrt(dot3(R2, R2));
    double c = a * b * (a * b + dot3(R1, R2));
    cross(R1, R2, cr);
    for (int m = 0; m < 3; m++) {
      double ub = (a + b) / c * cr[m];
      ub = ub * p->quant_circ / 4 / QO_PI;
      u[m] = u[m] + ub;
    }
    W->evals++;
  } else if (theta < p->tree_theta) {
    double v[3], ub[3];
    for (int c = 0; c < 3; c++) v[c] = xi[c] - (t->cent[c] + shift[c]);
    double d3 = dist * dist * dist;
    double d2 = dist * dist;
    double d5 = d2 * d2 * dist;
    cross(t->circ, v, ub);
    for (int m = 0; m < 3; m++) ub[m] = ub[m] / d3;
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < 3; l++) {
        double vc = v[0] * t->Cij[0][l];
        vc = vc + v[1] * t->Cij[1][l];
        vc = vc + v[2] * t->Cij[2][l];
        for (int m = 0; m < 3; m++) ub[m] = ub[m] - levi(m, k, l) * t->Cij[k][l] / d3;
        for (int m = 0; m < 3; m++) ub[m] = ub[m] + 3 * levi(m, k, l) * v[k] * vc / d5;
      }
    for (int m = 0; m < 3; m++) u[m] = u[m] + ub[m] * p->quant_circ / 4. / QO_PI;
    W->evals++;
  } else {
    for (int k = 0; k < 8; k++) tree_walk(W, t->child[k], shift, u);
  }
}

/* --------------------------------------------------------- biot_savart */
/* biot_savart, src/timestep.f90:462-482 (shift==NULL) and biot_savart_shift,
 * src/timestep.f90:485-507 */
static void biot_savart(const qo_params *p, int n, int i, const double *x,
                        const double *gi, const int *infront, const int *behind,
                        const double *shift, double *u) {
  const double *xi = x + 3 * i;
  for (int j = 0; j < n; j++) {
    if (infront[j] == 0) continue;
    if (shift == NULL) {
      if (i == j || behind[i] == j + 1) continue;
    } else {
      if (behind[i] == j + 1) continue;
    }
    const double *xj = x + 3 * j, *gj = gi + 3 * j;
    double d[3], s[3], ub[3];
    double a, b, c;
    if (shift == NULL) {
      for (int k = 0; k < 3; k++) d[k] = xj[k] - xi[k];
      a = sq(xj[0] - xi[0]) + sq(xj[1] - xi[1]) + sq(xj[2] - xi[2]); /* distfsq(j,i) */
    } else {
      double xs[3];
      for (int k = 0; k < 3; k++) xs[k] = xj[k] + shift[k];
      for (int k = 0; k < 3; k++) d[k] = xs[k] - xi[k];
      a = sq(xi[0] - xs[0]) + sq(xi[1] - xs[1]) + sq(xi[2] - xs[2]);
    }
    for (int k = 0; k < 3; k++) s[k] = gj[k] - xj[k];
    b = 2. * dot3(d, s);
    c = sq(gj[0] - xj[0]) + sq(gj[1] - xj[1]) + sq(gj[2] - xj[2]);
    if (4 * a * c - b * b == 0) continue;
    cross(d, s, ub);
    double disc = 4 * a * c - b * b;
    double fac = (2 * c + b) / sqrt(a + b + c) - (b / sqrt(a));
    for (int k = 0; k < 3; k++) {
      ub[k] = ub[k] * p->quant_circ / ((2 * QO_PI) * disc);
      ub[k] = ub[k] * fac;
      u[k] = u[k] + ub[k];
    }
  }
}

/* The list of image shifts in the reference's loop order
 * (src/timestep.f90:235-257, 283-305). */
static int image_shifts(const qo_params *p, double *sh) {
  int m = 0;
  double L = p->box_size;
  if (p->boundary == 1) {
    for (int a = -1; a <= 1; a++)
      for (int b = -1; b <= 1; b++)
        for (int c = -1; c <= 1; c++) {
          if (a == 0 && b == 0 && c == 0) continue;
          sh[3 * m] = a * L; sh[3 * m + 1] = b * L; sh[3 * m + 2] = c * L; m++;
        }
  } else if (p->boundary == 2) {
    for (int b = -1; b <= 1; b++)
      for (int c = -1; c <= 1; c++) {
        if (b == 0 && c == 0) continue;
        sh[3 * m] = 0.; sh[3 * m + 1] = b * L; sh[3 * m + 2] = c * L; m++;
      }
  } else if (p->boundary == 3) {
    for (int c = -1; c <= 1; c++) {
      if (c == 0) continue;
      sh[3 * m] = 0.; sh[3 * m + 1] = 0.; sh[3 * m + 2] = c * L; m++;
    }
  }
  return m;
}

/*
 * calc_velocity for one point, src/timestep.f90:180-309 (Off, LIA, BS and
 * Tree arms; mutual friction, forcing, hyperviscosity, mirror, sticky and
 * Hamiltonian terms are off at the run.in defaults and are not restated).
 * Returns 0, or -1 on the tree singularity (src/tree.f90:372-376).
 */
static int calc_velocity(const qo_params *p, int n, int i, const double *x,
                         const int *infront, const int *behind, const double *gi,
                         const double *gb, const double *gii, const double *gbb,
                         const qo_tree *T, double *u, double *u_li, double *u_bs,
                         long long *evals) {
  const double *xi = x + 3 * i;
  const double *Gi = gi + 3 * i, *Gb = gb + 3 * i, *Gii = gii + 3 * i, *Gbb = gbb + 3 * i;
  double fd[3], fdd[3], cr[3], ubs[3];
  u[0] = u[1] = u[2] = 0.;
  if (u_li) u_li[0] = u_li[1] = u_li[2] = 0.;
  if (u_bs) u_bs[0] = u_bs[1] = u_bs[2] = 0.;
  if (p->velocity == 0) return 0;
  deriv1(p, xi, Gi, Gb, Gii, Gbb, fd);
  deriv2(p, xi, Gi, Gb, Gii, Gbb, fdd);
  double beta;
  if (p->velocity == 1) {
    if (p->fixed_lia_beta) {
      beta = 1.3E-3;
    } else {
      double curv = sqrt(dot3(fdd, fdd));
      if (curv < QO_EPS)
        curv = QO_EPS;
      else
        curv = 1. / curv;
      beta = (p->quant_circ / (4. * QO_PI)) * log(curv / p->corea);
    }
    cross(fd, fdd, cr);
    for (int c = 0; c < 3; c++) u[c] = beta * cr[c];
    return 0;
  }
  beta = (p->quant_circ / (4. * QO_PI)) *
         log((1.21 / p->corea) * sqrt(dist_gen(xi, Gi) * dist_gen(xi, Gb)));
  cross(fd, fdd, cr);
  for (int c = 0; c < 3; c++) u[c] = beta * cr[c];
  if (u_li) for (int c = 0; c < 3; c++) u_li[c] = u[c];
  double sh[26 * 3];
  int nimg = image_shifts(p, sh);
  int status = 0;
  if (p->velocity == 2) {
    ubs[0] = ubs[1] = ubs[2] = 0.;
    biot_savart(p, n, i, x, gi, infront, behind, NULL, ubs);
    for (int c = 0; c < 3; c++) u[c] = u[c] + ubs[c];
    if (u_bs) for (int c = 0; c < 3; c++) u_bs[c] = ubs[c];
    if (nimg) {
      ubs[0] = ubs[1] = ubs[2] = 0.;
      for (int m = 0; m < nimg; m++) biot_savart(p, n, i, x, gi, infront, behind, sh + 3 * m, ubs);
      for (int c = 0; c < 3; c++) u[c] = u[c] + ubs[c];
      if (u_bs) for (int c = 0; c < 3; c++) u_bs[c] = u_bs[c] + ubs[c];
    }
  } else {
    walk_ctx W = {p, i, xi, infront, behind, 0, 0};
    double zero[3] = {0., 0., 0.};
    ubs[0] = ubs[1] = ubs[2] = 0.;
    tree_walk(&W, T->root, zero, ubs);
    for (int c = 0; c < 3; c++) u[c] = u[c] + ubs[c];
    if (u_bs) for (int c = 0; c < 3; c++) u_bs[c] = ubs[c];
    if (nimg) {
      ubs[0] = ubs[1] = ubs[2] = 0.;
      for (int m = 0; m < nimg; m++) tree_walk(&W, T->root, sh + 3 * m, ubs);
      for (int c = 0; c < 3; c++) u[c] = u[c] + ubs[c];
      if (u_bs) for (int c = 0; c < 3; c++) u_bs[c] = u_bs[c] + ubs[c];
    }
    if (evals) *evals += W.evals;
    status = W.status;
  }
  return status;
}

/*
 * Velocity of the listed targets (all active slots when targets==NULL).
 * Returns 0, or -1 if any tree evaluation hit the singularity.  nthreads>1
 * runs targets in parallel; each target's sum stays sequential, so results
 * do not depend on the thread count.
 */
int qo_velocity(const qo_params *p, int n, const double *x, const int *infront,
                const int *behind, const double *gi, const double *gb,
                const double *gii, const double *gbb, const qo_tree *T,
                int ntargets, const int *targets, double *u, double *u_li,
                double *u_bs, long long *evals, int nthreads) {
  int nt = targets ? ntargets : n;
  int status = 0;
  long long ev = 0;
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads) reduction(+ : ev) reduction(min : status)
#endif
  for (int q = 0; q < nt; q++) {
    int i = targets ? targets[q] : q;
    if (infront[i] == 0) continue;
    long long e = 0;
    int s = calc_velocity(p, n, i, x, infront, behind, gi, gb, gii, gbb, T, u + 3 * q,
                          u_li ? u_li + 3 * q : NULL, u_bs ? u_bs + 3 * q : NULL, &e);
    ev += e;
    if (s < status) status = s;
  }
  if (evals) {
    /* construct_tree sets eval_counter=2*count(active) for Tree (src/tree.f90:77-78) */
    long long base = 0;
    if (p->velocity == 3) {
      for (int i = 0; i < n; i++) if (infront[i] > 0) base += 2;
    }
    *evals = base + ev;
  }
  return status;
}

/* ------------------------------------------------------------- time step */
/* pmotion AB ladder, src/timestep.f90:48-71 (dt_adapt off) */
void qo_pmotion_ab(double dt, int n, double *x, const double *u, double *u1,
                   double *u2, double *u3, const int *infront) {
  const double three_twos = 3. / 2., one_half = 1. / 2.;
  const double twenty_three_twelve = 23. / 12., four_thirds = 4. / 3.,
               five_twelths = 5. / 12.;
  for (int i = 0; i < n; i++) {
    if (infront[i] == 0) continue;
    double *X = x + 3 * i, *U1 = u1 + 3 * i, *U2 = u2 + 3 * i, *U3 = u3 + 3 * i;
    const double *U = u + 3 * i;
    int z1 = (fabs(U1[0]) == 0 && fabs(U1[1]) == 0 && fabs(U1[2]) == 0);
    int z2 = (fabs(U2[0]) == 0 && fabs(U2[1]) == 0 && fabs(U2[2]) == 0);
    int z3 = (fabs(U3[0]) == 0 && fabs(U3[1]) == 0 && fabs(U3[2]) == 0);
    for (int c = 0; c < 3; c++) {
      if (z1)
        X[c] = X[c] + dt * U[c];
      else if (z2)
        X[c] = X[c] + three_twos * dt * U[c] - one_half * dt * U1[c];
      else if (z3)
        X[c] = X[c] + twenty_three_twelve * dt * U[c] - four_thirds * dt * U1[c] +
               five_twelths * dt * U2[c];
      else
        X[c] = X[c] + dt * (55. * U[c] - 59. * U1[c] + 37. * U2[c] - 9. * U3[c]) / 24.;
    }
    for (int c = 0; c < 3; c++) {
      U3[c] = U2[c];
      U2[c] = U1[c];
      U1[c] = U[c];
    }
  }
}

/* ------------------------------------------------------ candidate search */
typedef struct {
  int i;
  const double *xi;
  const int *infront, *behind;
  int *closest;
  double *closestd;
} close_ctx;

/* closest_tree, src/tree.f90:237-278 (mirror branch out of scope) */
static void closest_tree(close_ctx *C, const qo_node *t) {
  int i = C->i;
  if (C->infront[i] == 0) return;
  if (t->pcount == 0) return;
  const double *xi = C->xi;
  double dist = sqrt(sq(xi[0] - t->cent[0]) + sq(xi[1] - t->cent[1]) + sq(xi[2] - t->cent[2]));
  double theta = t->width / dist;
  if (t->pcount == 1 || theta < .5) {
    if (dist < *C->closestd) {
      if (t->pcount > 1) {
        *C->closest = 0; /* j is read but unused on this branch */
      } else {
        int j = C->behind[t->first_infront - 1]; /* f(parray(1)%infront)%behind */
        if ((i + 1 != j) && (C->infront[i] != j) && (C->behind[i] != j)) {
          *C->closest = j;
          *C->closestd = dist;
        }
      }
    }
  } else {
    for (int k = 0; k < 8; k++) closest_tree(C, t->child[k]);
  }
}

/* pclose_tree, src/tree.f90:219-234.  closest is in/out (never reset). */
void qo_pclose_tree(const qo_tree *T, int n, const double *x, const int *infront,
                    const int *behind, int *closest, double *closestd, int nthreads) {
#ifdef _OPENMP
  if (nthreads < 1) nthreads = 1;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads)
#endif
  for (int i = 0; i < n; i++) {
    closestd[i] = 100.;
    if (infront[i] == 0) continue;
    close_ctx C = {i, x + 3 * i, infront, behind, closest + i, closestd + i};
    closest_tree(&C, T->root);
  }
}

/* pclose (no tree), src/line.f90:205-234 */
void qo_pclose(int n, const double *x, const int *infront, const int *behind,
               int *closest, double *closestd) {
  for (int i = 0; i < n; i++) {
    if (infront[i] == 0) continue;
    closestd[i] = 100.;
    for (int j = 0; j < n; j++) {
      if (infront[j] == 0) continue;
      if ((i != j) && (infront[i] != j + 1) && (behind[i] != j + 1)) {
        double dist = sqrt(sq(x[3 * i] - x[3 * j]) + sq(x[3 * i + 1] - x[3 * j + 1]) +
                           sq(x[3 * i + 2] - x[3 * j + 2]));
        if (dist < closestd[i]) {
          closest[i] = j + 1;
          closestd[i] = dist;
        }
      }
    }
  }
}

/* ------------------------------------------------------------------ energy */
/* energy_info, src/diagnostic.f90:259-280 */
double qo_energy(const qo_params *p, int n, const double *x, const double *u,
                 const int *infront, const double *gi, const double *gb,
                 const double *gii, const double *gbb) {
  double energy = 0.;
  for (int i = 0; i < n; i++) {
    if (infront[i] == 0) continue;
    int a = infront[i] - 1;
    double sd[3], sdi[3], c1[3], c2[3];
    deriv1(p, x + 3 * i, gi + 3 * i, gb + 3 * i, gii + 3 * i, gbb + 3 * i, sd);
    deriv1(p, x + 3 * a, gi + 3 * a, gb + 3 * a, gii + 3 * a, gbb + 3 * a, sdi);
    cross(x + 3 * i, sd, c1);
    cross(x + 3 * a, sdi, c2);
    energy = energy + 0.5 * dist_gen(x + 3 * i, gi + 3 * i) *
                          (dot3(u + 3 * i, c1) + dot3(u + 3 * a, c2));
  }
  return energy * (p->quant_circ);
}

/* -------------------------------------------------------------- full step */
/*
 * One pass of the loop body of src/run.f90:36-169 restricted to the path:
 * ghostp, construct_tree (tree_theta>0), pmotion or pmotion_RK3, the
 * candidate search (pclose_tree or pclose, every recon_shots steps), ghostp
 * and the boundary wrap.  Insertion, removal and reconnection surgery are
 * not part of the path and are not run.  closest/closestd may be NULL to skip
 * the search.  Returns 0, or a negative status.
 */
int qo_step(const qo_params *p, int n, double *x, const int *infront, const int *behind,
            double *u, double *u1, double *u2, double *u3, double *gi, double *gb,
            double *gii, double *gbb, int runge_kutta, int *closest, double *closestd,
            long long *evals, int nthreads) {
  int status = 0;
  qo_ghosts(p, n, x, infront, behind, gi, gb, gii, gbb);
  qo_tree *T = NULL;
  if (p->tree_theta > 0) {
    T = qo_tree_build(p, n, x, gi, infront);
    if (T->status) { qo_tree_free(T); return -2; }
  }
  if (!runge_kutta) {
    status = qo_velocity(p, n, x, infront, behind, gi, gb, gii, gbb, T, 0, NULL, u, NULL,
                         NULL, evals, nthreads);
    qo_pmotion_ab(p->dt, n, x, u, u1, u2, u3, infront);
  } else {
    /* pmotion_RK3, src/timestep.f90:95-176 */
    double dt = p->dt;
    for (int stage = 0; stage < 3; stage++) {
      if (stage > 0) {
        qo_ghosts(p, n, x, infront, behind, gi, gb, gii, gbb);
        if (T) {
          qo_tree_free(T);
          T = qo_tree_build(p, n, x, gi, infront);
          if (T->status) { qo_tree_free(T); return -2; }
        }
      }
      int s = qo_velocity(p, n, x, infront, behind, gi, gb, gii, gbb, T, 0, NULL, u, NULL,
                          NULL, evals, nthreads);
      if (s < status) status = s;
      for (int i = 0; i < n; i++) {
        if (infront[i] == 0) continue;
        for (int c = 0; c < 3; c++) {
          double uu = u[3 * i + c];
          if (stage == 0) u1[3 * i + c] = uu * dt;
          else if (stage == 1) u1[3 * i + c] = -(2. / 3.) * u1[3 * i + c] + uu * dt;
          else u1[3 * i + c] = -u1[3 * i + c] + uu * dt;
        }
      }
      for (int i = 0; i < n; i++) {
        if (infront[i] == 0) continue;
        for (int c = 0; c < 3; c++) {
          if (stage == 0) x[3 * i + c] = x[3 * i + c] + (u1[3 * i + c] / 3.);
          else if (stage == 1) x[3 * i + c] = x[3 * i + c] + u1[3 * i + c];
          else x[3 * i + c] = x[3 * i + c] + 0.5 * u1[3 * i + c];
        }
      }
    }
  }
  if (closest && closestd) {
    if (T)
      qo_pclose_tree(T, n, x, infront, behind, closest, closestd, nthreads);
    else
      qo_pclose(n, x, infront, behind, closest, closestd);
  }
  qo_ghosts(p, n, x, infront, behind, gi, gb, gii, gbb);
  if (p->boundary >= 1 && p->boundary <= 3) qo_enforce_periodic(p, n, x, infront);
  if (T) qo_tree_free(T);
  return status;
}

/* timestep_check bound, src/initial.f90:606-622 */
double qo_dt_max(const qo_params *p) {
  double delta_min = p->delta / 2.;
  return fabs((sq(delta_min)) / (p->quant_circ * log(delta_min / (QO_PI * p->corea))));
}

void qo_set_depth_cap(int cap) { g_depth_cap = cap; }

/* ------------------------------------------------ insertion and removal */
/* The point state the line operations read and write (arrays of cap slots). */
typedef struct {
  double *x, *u, *u1, *u2, *u3, *gi, *gb, *gii, *gbb, *u_li, *u_bs, *closestd;
  int *infront, *behind, *closest;
} qo_state;

/* get_ghost_p for one slot, src/periodic.f90:23-165 */
static void ghost_one(const qo_params *p, int i, const qo_state *S) {
  int a = S->infront[i] - 1, b = S->behind[i] - 1;
  int aa = S->infront[a] - 1, bb = S->behind[b] - 1;
  double *G[4] = {S->gi + 3 * i, S->gb + 3 * i, S->gii + 3 * i, S->gbb + 3 * i};
  int src[4] = {a, b, aa, bb};
  for (int k = 0; k < 4; k++)
    for (int c = 0; c < 3; c++) G[k][c] = S->x[3 * src[k] + c];
  int lo = 3;
  if (p->boundary == 1) lo = 0;
  else if (p->boundary == 2) lo = 1;
  else if (p->boundary == 3) lo = 2;
  for (int axis = lo; axis < 3; axis++)
    for (int k = 0; k < 4; k++) unwrap(p, S->x + 3 * i, G[k], axis);
}

/* clear_particle, src/general.f90:11-22 (u3, delta and t_recon are kept) */
static void clear_particle(qo_state *S, int i) {
  for (int c = 0; c < 3; c++) {
    S->x[3 * i + c] = 0.; S->u[3 * i + c] = 0.; S->u1[3 * i + c] = 0.; S->u2[3 * i + c] = 0.;
    S->gi[3 * i + c] = 0.; S->gb[3 * i + c] = 0.; S->gii[3 * i + c] = 0.; S->gbb[3 * i + c] = 0.;
    S->u_li[3 * i + c] = 0.; S->u_bs[3 * i + c] = 0.;
  }
  S->infront[i] = 0; S->behind[i] = 0;
  S->closest[i] = 0; S->closestd[i] = 0.;
}

/* pinsert, src/line.f90:18-106 (delta_adapt, mirror and particles_only off).
 * *pcount grows by the points appended past the last slot; returns the number
 * of points inserted, or -1 when more than cap slots would be needed.  The
 * ghosts read are the stored ones (computed before the move, refreshed only
 * for the slots an insertion touches), as in the reference.  A slot appended
 * to the array gets u3 = 0, closest = 0 and zero velocities (the reference
 * leaves those components of a new array element undefined; none of them
 * enters a result before it is overwritten). */
int qo_pinsert(const qo_params *p, int *pcount, int cap, qo_state *S) {
  int old_pcount = *pcount, inserted = 0;
  for (int i = 0; i < old_pcount; i++) {
    if (S->infront[i] == 0) continue;
    double disti = dist_gen(S->x + 3 * i, S->gi + 3 * i);
    if (disti > 1. * p->delta) {
      int par_new = -1;
      for (int k = 0; k < *pcount; k++)
        if (S->infront[k] == 0) { par_new = k; break; }   /* minloc(f(:)%infront) */
      if (par_new < 0) {
        if (*pcount >= cap) return -1;
        par_new = *pcount;
        *pcount = *pcount + 1;
        for (int c = 0; c < 3; c++) {
          S->u3[3 * par_new + c] = 0.; S->u_li[3 * par_new + c] = 0.; S->u_bs[3 * par_new + c] = 0.;
        }
        S->closest[par_new] = 0; S->closestd[par_new] = 0.;
      }
      double fdd[3];
      deriv2(p, S->x + 3 * i, S->gi + 3 * i, S->gb + 3 * i, S->gii + 3 * i, S->gbb + 3 * i, fdd);
      double curv = sqrt(dot3(fdd, fdd));
      double *xn = S->x + 3 * par_new;
      const double *xi = S->x + 3 * i, *gi = S->gi + 3 * i;
      if (curv > 1E-5) {
        curv = 1. / curv;
        if (curv * curv - 0.25 * (disti * disti) > 0.) {
          double f = (sqrt(curv * curv - 0.25 * (disti * disti)) - curv) * curv;
          for (int c = 0; c < 3; c++) xn[c] = 0.5 * (xi[c] + gi[c]) + f * fdd[c];
        } else {
          for (int c = 0; c < 3; c++) xn[c] = 0.5 * (xi[c] + gi[c]);
        }
      } else {
        for (int c = 0; c < 3; c++) xn[c] = 0.5 * (xi[c] + gi[c]);
      }
      int a = S->infront[i] - 1;
      for (int c = 0; c < 3; c++) {
        S->u[3 * par_new + c] = 0.5 * (S->u[3 * i + c] + S->u[3 * a + c]);
        S->u1[3 * par_new + c] = 0.;
        S->u2[3 * par_new + c] = 0.;
      }
      S->behind[par_new] = i + 1;
      S->infront[par_new] = S->infront[i];
      ghost_one(p, par_new, S);
      S->behind[a] = par_new + 1;
      ghost_one(p, a, S);
      S->infront[i] = par_new + 1;
      ghost_one(p, i, S);
      inserted++;
    }
  }
  return inserted;
}

/* loop_killer, src/reconnection.f90:421-461: a loop of fewer than 5 points
 * is cleared (the log of small loops is output only). */
static int loop_killer(qo_state *S, int pcount, int particle) {
  int counter = 1, next = particle;
  for (int k = 0; k < pcount; k++) {
    next = S->infront[next] - 1;
    if (next == particle || next < 0) break;  /* next < 0: a cleared slot (a broken loop) */
    counter++;
  }
  if (counter >= 5) return 0;
  next = particle;
  for (int k = 0; k < pcount; k++) {
    int store_next = S->infront[next] - 1;
    clear_particle(S, next);
    next = store_next;
    if (next == particle || next < 0) break;
  }
  return counter;
}

/* premove, src/line.f90:112-161 (mirror, phonon emission and recon_info off;
 * every point's delta factor is 1, as pinsert leaves it).  distf is taken on
 * raw positions, without periodic unwrapping, as in the reference.  Returns
 * the number of points removed (loops cleared by loop_killer included). */
int qo_premove(const qo_params *p, int pcount, qo_state *S) {
  int removed = 0;
  for (int i = 0; i < pcount; i++) {
    if (S->infront[i] == 0) continue;
    int a = S->infront[i] - 1, aa = S->infront[a] - 1;
    const double *xi = S->x + 3 * i, *xj = S->x + 3 * aa;
    double distii = sqrt(sq(xi[0] - xj[0]) + sq(xi[1] - xj[1]) + sq(xi[2] - xj[2]));
    if (distii < .499 * p->delta * (1. + 1.)) {
      S->behind[aa] = i + 1;
      S->infront[i] = aa + 1;
      clear_particle(S, a);
      removed += 1 + loop_killer(S, pcount, i);
    }
  }
  return removed;
}

/* norm_tanf, src/general.f90:94-107: get_deriv_1 on the stored ghosts, normalised */
static void norm_tanf(const qo_params *p, const qo_state *S, int i, double *t) {
  deriv1(p, S->x + 3 * i, S->gi + 3 * i, S->gb + 3 * i, S->gii + 3 * i, S->gbb + 3 * i, t);
  double length = sqrt(sq(t[0]) + sq(t[1]) + sq(t[2]));
  for (int c = 0; c < 3; c++) t[c] = t[c] / length;
}

/* precon_original, src/reconnection.f90:145-254 (recon_info and recon_time_info
 * off).  Reads closest/closestd of the last candidate search and the stored
 * ghosts; returns the number of reconnections. */
int qo_precon(const qo_params *p, int pcount, qo_state *S) {
  int count = 0;
  for (int i = 0; i < pcount; i++) {
    if (S->infront[i] == 0) continue;
    int pari = S->infront[i] - 1, parb = S->behind[i] - 1;
    if (!((S->closestd[i] < p->delta / 2.) && (S->closestd[i] > QO_EPS))) continue;
    int j = S->closest[i] - 1;
    if (j == pari) continue;
    if (j == parb) continue;
    if (j == -1) continue;
    if (S->infront[j] == 0) continue;
    int parjb = S->behind[j] - 1;
    double t1[3], t2[3];
    norm_tanf(p, S, i, t1);
    norm_tanf(p, S, j, t2);
    double dot_val = t1[0] * t2[0] + t1[1] * t2[1] + t1[2] * t2[2];
    if (dot_val > 0.9) continue;
    const double *xi = S->x + 3 * i, *xj = S->x + 3 * j;
    double l_before = dist_gen(xi, S->gi + 3 * i) + dist_gen(xi, S->gb + 3 * i) +
                      dist_gen(xj, S->gi + 3 * j) + dist_gen(xj, S->gb + 3 * j);
    double l_after = dist_gen(xi, S->gb + 3 * i) + dist_gen(xi, xj) +
                     dist_gen(xj, S->gi + 3 * j) + dist_gen(S->x + 3 * pari, S->x + 3 * parjb);
    if (l_after <= l_before) {
      count++;
      S->infront[parjb] = pari + 1;
      S->behind[pari] = parjb + 1;
      S->infront[i] = j + 1;
      S->behind[j] = i + 1;
      loop_killer(S, pcount, pari);
      loop_killer(S, pcount, i);
    }
  }
  return count;
}

/* ------------------------------------------------ tree_walk_general */
/* tree_walk_general, src/tree.f90:425-488 (hollow_mesh_core off): the velocity
 * at an arbitrary point from the tree, as mesh_velocity uses it
 * (src/timestep.f90:374-452).  The leaf term is divided by 4 pi and the
 * far-field term is not, and neither is multiplied by quant_circ: the
 * reference's own scaling, kept as it is. */
static void walk_general(const qo_params *p, const qo_node *t, const double *x,
                         const double *shift, double *u, long long *evals) {
  if (!t || t->pcount == 0) return;
  double dist = sqrt(sq(x[0] - (t->cent[0] + shift[0])) + sq(x[1] - (t->cent[1] + shift[1])) +
                     sq(x[2] - (t->cent[2] + shift[2])));
  if (dist < QO_EPS) return;
  double theta = t->width / dist;
  if (t->pcount == 1) {
    double v1[3], v2[3], cr[3];
    for (int c = 0; c < 3; c++) {
      v1[c] = t->cent[c] + shift[c] - x[c];
      v2[c] = t->cent[c] + t->circ[c] + shift[c] - x[c];
    }
    double a = sqrt(dot3(v1, v1)), b = sqrt(dot3(v2, v2));
    double c = a * b * (a * b + dot3(v1, v2));
    cross(v1, v2, cr);
    for (int m = 0; m < 3; m++) {
      double ub = (a + b) / c * cr[m];
      u[m] = u[m] + ub / 4 / QO_PI;
    }
    (*evals)++;
  } else if (theta < p->tree_theta) {
    double v[3], ub[3];
    for (int c = 0; c < 3; c++) v[c] = x[c] - (t->cent[c] + shift[c]);
    double d3 = dist * dist * dist;
    double d2 = dist * dist;
    double d5 = d2 * d2 * dist;
    cross(t->circ, v, ub);
    for (int m = 0; m < 3; m++) ub[m] = ub[m] / d3;
    for (int k = 0; k < 3; k++)
      for (int l = 0; l < 3; l++) {
        double vc = v[0] * t->Cij[0][l];
        vc = vc + v[1] * t->Cij[1][l];
        vc = vc + v[2] * t->Cij[2][l];
        for (int m = 0; m < 3; m++) ub[m] = ub[m] - levi(m, k, l) * t->Cij[k][l] / d3;
        for (int m = 0; m < 3; m++) ub[m] = ub[m] + 3 * levi(m, k, l) * v[k] * vc / d5;
      }
    for (int m = 0; m < 3; m++) u[m] = u[m] + ub[m];
    (*evals)++;
  } else {
    for (int k = 0; k < 8; k++) walk_general(p, t->child[k], x, shift, u, evals);
  }
}

/* The Tree arm of mesh_velocity for m points: the unshifted tree, then the
 * images of the boundary in the reference's loop order. */
long long qo_field_velocity_tree(const qo_params *p, const qo_tree *T, int m, const double *pts,
                                 double *u) {
  double sh[27 * 3];
  int ns = image_shifts(p, sh);
  long long evals = 0;
  for (int q = 0; q < m; q++) {
    double *uq = u + 3 * q;
    uq[0] = uq[1] = uq[2] = 0.;
    const double zero[3] = {0., 0., 0.};
    walk_general(p, T->root, pts + 3 * q, zero, uq, &evals);
    for (int s = 0; s < ns; s++) walk_general(p, T->root, pts + 3 * q, sh + 3 * s, uq, &evals);
  }
  return evals;
}

/* ------------------------------------------------ biot_savart_general */
/* biot_savart_general (shift == NULL) and biot_savart_general_shift,
 * src/timestep.f90:516-563: the velocity at an arbitrary point x from every
 * active segment j -> ghosti(j) (no skip rule), added into u, in the
 * reference's operation order. */
static void bs_general(const qo_params *p, int n, const double *xs, const double *gi,
                       const int *infront, const double *x, const double *shift, double *u) {
  for (int i = 0; i < n; i++) {
    if (infront[i] == 0) continue;
    const double *xi = xs + 3 * i, *gj = gi + 3 * i;
    double xsh[3], d[3], s[3], ub[3];
    for (int k = 0; k < 3; k++) xsh[k] = shift ? xi[k] + shift[k] : xi[k];
    double a = dist_gen_sq(x, xsh);
    for (int k = 0; k < 3; k++) { d[k] = xsh[k] - x[k]; s[k] = gj[k] - xi[k]; }
    double b = 2. * dot3(d, s);
    double c = dist_gen_sq(gj, xi);
    if ((4 * a * c - b * b) == 0) continue;
    cross(d, s, ub);
    for (int k = 0; k < 3; k++) ub[k] = ub[k] * p->quant_circ / ((2 * QO_PI) * (4 * a * c - b * b));
    double fac = (2 * c + b) / sqrt(a + b + c) - (b / sqrt(a));
    for (int k = 0; k < 3; k++) ub[k] = ub[k] * fac;
    for (int k = 0; k < 3; k++) u[k] = u[k] + ub[k];
  }
}

/* The BS arm of mesh_velocity (src/timestep.f90:393-416) at m points: the
 * unshifted sum, then the boundary's images in the reference's loop order,
 * into one running sum per point. */
void qo_field_velocity(const qo_params *p, int n, const double *xs, const double *gi,
                       const int *infront, int m, const double *pts, double *u) {
  double sh[27 * 3];
  int ns = image_shifts(p, sh);
  for (int q = 0; q < m; q++) {
    double *uq = u + 3 * q;
    uq[0] = uq[1] = uq[2] = 0.;
    bs_general(p, n, xs, gi, infront, pts + 3 * q, NULL, uq);
    for (int s = 0; s < ns; s++) bs_general(p, n, xs, gi, infront, pts + 3 * q, sh + 3 * s, uq);
  }
}
