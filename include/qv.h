/*
 * qv.h -- C ABI of the B200 velocity-and-timestep path for Qvort filaments.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (QV_OK = 0, negative = error; nothing throws across the ABI) and
 * is synchronous at return unless its name ends in _async.  A context owns the
 * device buffers of one filament system; calls on one context must not
 * overlap (it is not re-entrant).  Work is issued on the context's stream.
 *
 * Data conventions follow the reference's point array f(:) (src/cdata.f90:20-39):
 *   n slots; positions and velocities are interleaved x[3*i+c] (the column-major
 *   layout of a Fortran real(c_double) :: x(3,n)); infront/behind hold 1-based
 *   slot indices and infront==0 marks an empty slot that every loop skips
 *   (src/timestep.f90:43).
 *
 * Each entry point cites the reference routine (file:line, within abag/qvort)
 * whose call it replaces.
 */
#ifndef QV_H
#define QV_H
#ifdef __cplusplus
extern "C" {
#endif

#define QV_OK 0
#define QV_ERR_ARG (-1)        /* bad argument or size */
#define QV_ERR_CUDA (-2)       /* a CUDA call failed, or a device-side copy did not complete
                                  within its bounded wait (the outputs of that call are then
                                  undefined); see qv_last_error */
#define QV_ERR_SINGULAR (-3)   /* tree singularity (src/tree.f90:372-376) */
#define QV_ERR_TREE_DEPTH (-4) /* octree deeper than QV_MAX_DEPTH (coincident points) */
#define QV_ERR_STATE (-5)      /* call out of order (no points, no tree, ...) */
#define QV_ERR_NOMEM (-6)      /* device allocation failed */
#define QV_ERR_UNSUPPORTED (-7)/* a run.in option outside this path (mirror, forcing, ...) */
#define QV_ERR_NAN (-8)        /* NaN in the positions of any slot at the end of a step
                                  (NAN_finder, src/general.f90:253-280; run.f90:168) */
#define QV_ERR_NOALLOC_LIMIT (-9) /* more slots than QV_NOALLOC_MAX_POINTS */

#define QV_MAX_DEPTH 64

/* boundary (src/initial.f90:106-136) */
#define QV_BC_OPEN 0
#define QV_BC_PERIODIC 1
#define QV_BC_OPENX 2  /* periodic in y,z */
#define QV_BC_OPENXY 3 /* periodic in z */
/* velocity (src/cdata.f90:489-491) */
#define QV_VEL_OFF 0
#define QV_VEL_LIA 1
#define QV_VEL_BS 2
#define QV_VEL_TREE 3
/* arithmetic of the non-local sums */
#define QV_PREC_FP64 0  /* FP64 throughout (the reference's arithmetic) */
#define QV_PREC_MIXED 1 /* FP32 pair terms, FP64 recentring, compensated sums */

/* run.in parameters used by the path (src/cdata.f90:196-416) */
typedef struct qv_params {
  double quant_circ;          /* quant_circ, default 9.97e-4 */
  double corea;               /* corea, default 8.244023e-9 */
  double box_size;            /* box_size */
  double delta;               /* delta */
  double dt;                  /* dt */
  double tree_theta;          /* tree_theta (0: direct sum, pclose) */
  int boundary;               /* QV_BC_* */
  int velocity;               /* QV_VEL_* */
  int deriv_order;            /* 2 ('second') or 4 ('fourth') */
  int tree_extra_correction;  /* tree_extra_correction, default 1 */
  int fixed_lia_beta;         /* fixed_LIA_beta */
  int precision;              /* QV_PREC_* */
  int runge_kutta;            /* runge_kutta */
  int recon_shots;            /* recon_shots, default 1 */
  int line_ops;               /* 0 (default): qv_step leaves the line operations to the
                                 caller (qv_pinsert, qv_precon, qv_premove); 1: qv_step
                                 runs pinsert after the update and premove after the
                                 candidate search (src/run.f90:59-72 with switch_off_recon
                                 true); 2: also precon_original between the search and
                                 premove (the reference's default loop) */
} qv_params;

typedef struct qv_ctx qv_ctx;

/* Fill *p with the reference's run.in defaults (src/cdata.f90:196-416). */
int qv_default_params(qv_params *p);

/* Create / destroy a context.  Replaces nothing: the reference keeps state in
 * module variables (src/cdata.f90).  Every launch and copy of the context goes
 * to `stream`; NULL makes the context create a private non-blocking stream,
 * which is not ordered with any other stream, so a caller that hands the
 * context device buffers written by work on the legacy default stream passes
 * cudaStreamLegacy ((void *)0x1) instead of NULL. */
int qv_create(const qv_params *p, void *stream, qv_ctx **out);
int qv_destroy(qv_ctx *ctx);
int qv_set_params(qv_ctx *ctx, const qv_params *p);
const char *qv_last_error(const qv_ctx *ctx);

/* Gather of f(:)%x, f(:)%infront, f(:)%behind into the context (host
 * pointers).  Resets the AB history and closest to zero.  The links are
 * checked before the context takes anything (this, qv_set_state and
 * qv_step_exchange): they are uploaded to a staging buffer and a kernel tests
 * every infront/behind (and closest, where given) in 0..n, and an active slot
 * linking forwards and backwards to active slots; otherwise QV_ERR_ARG naming
 * the first offending slot, and the context's state is as it was. */
int qv_set_points(qv_ctx *ctx, int n, const double *x, const int *infront, const int *behind);
/* The same from device pointers (the torch harness); the links are the
 * caller's device arrays and are not checked. */
int qv_set_points_device(qv_ctx *ctx, int n, const double *x, const int *infront,
                         const int *behind);
/* f(:)%u1..u3 in/out (host; NULL means zero on set, skip on get). */
int qv_set_history(qv_ctx *ctx, const double *u1, const double *u2, const double *u3);
int qv_get_history(qv_ctx *ctx, double *u1, double *u2, double *u3);
/* f(:)%closest in/out; pclose_tree never resets it (src/tree.f90:225). */
int qv_set_closest(qv_ctx *ctx, const int *closest);
/* Scatter back f(:)%x and f(:)%u (host; NULL skips). */
int qv_get_points(qv_ctx *ctx, double *x, double *u);
/* Scatter back f(:)%closest and f(:)%closestd of the last candidate search. */
int qv_get_closest(qv_ctx *ctx, int *closest, double *closestd);

/* The per-point state a host copy of f(:) exchanges with the path each step
 * (src/cdata.f90:20-39): host arrays of 3n (vectors) or n (scalars) entries.
 * qv_set_state is qv_set_points + qv_set_history + qv_set_closest in one call
 * (u1..u3 or closest NULL: zeros; u and closestd are not read); qv_get_state
 * copies every non-NULL array back for the n slots in use (*n), or returns
 * QV_ERR_ARG with *n set when n exceeds cap (insertion grew the slot count:
 * the host grows its arrays and calls again).  One wait each. */
typedef struct qv_state {
  double *x, *u, *u1, *u2, *u3;
  int *infront, *behind, *closest;
  double *closestd;
} qv_state;
int qv_set_state(qv_ctx *ctx, int n, const qv_state *s);
int qv_get_state(qv_ctx *ctx, int cap, qv_state *s, int *n);
/* One iteration of the run.f90 loop (src/run.f90:41-93) with the host copy of
 * f(:): the same as qv_set_state(n, in), qv_step(itime), qv_get_state(cap,
 * out, n_out), with one wait.  The copies overlap the step as far as the data
 * allows: the AB history and closest go up on a side stream and the update
 * waits for them; everything but x comes back while the closing ghosts and
 * wrap run.  in and out may point at the same host arrays; none of them is
 * read or written after the call returns.  n_out > cap: QV_ERR_ARG with
 * *n_out set and out untouched (the step itself has run). */
int qv_step_exchange(qv_ctx *ctx, int itime, int n, const qv_state *in, int cap, qv_state *out,
                     int *n_out);
/* Device pointers of the context's arrays (valid until the next set_points). */
int qv_device_arrays(qv_ctx *ctx, double **x, double **u, int **infront, int **behind);

/* ghostp (src/periodic.f90:8-17): ghosts from positions and links. */
int qv_ghosts(qv_ctx *ctx);
int qv_get_ghosts(qv_ctx *ctx, double *gi, double *gb, double *gii, double *gbb);

/* construct_tree (src/tree.f90:44-80): the octree, bit-exact. */
int qv_build_tree(qv_ctx *ctx);
/* Number of nodes and depth of the last tree. */
int qv_tree_info(qv_ctx *ctx, int *nnodes, int *depth);
/* Non-empty nodes of the last tree in breadth-first order, children in the
 * fixed fbl..btr order (src/tree.f90:92-114); the same layout the oracle
 * exports.  Returns the node count, or -count when cap is too small. */
int qv_tree_export(qv_ctx *ctx, int cap, int *parent, int *digit, int *depth, double *pos,
                   double *width, int *pcount, double *cent, double *circ, double *Cij,
                   int *first);

/* The first loop of pmotion (src/timestep.f90:41-47) = calc_velocity
 * (src/timestep.f90:180-309) for every active point, LIA + Biot-Savart direct
 * sum or tree walk + periodic images.  Host outputs may be NULL; eval_count
 * receives the reference's eval_counter (src/tree.f90:63-79,393,413). */
int qv_velocity(qv_ctx *ctx, double *u, double *u_li, double *u_bs, long long *eval_count);

/* The second loop of pmotion (src/timestep.f90:48-71): the AB ladder on the
 * context's velocities, then the u3<-u2<-u1<-u shift. */
int qv_step_ab(qv_ctx *ctx);
/* pmotion_RK3 (src/timestep.f90:95-176): 3 velocity stages with ghost and
 * tree rebuilds between them. */
int qv_step_rk3(qv_ctx *ctx);
/* enforce_periodic and the yz / z variants (src/periodic.f90:188-214). */
int qv_enforce_periodic(qv_ctx *ctx);

/* pclose_tree (src/tree.f90:219-278) on the tree of the last build and the
 * current positions and links, or pclose (src/line.f90:205-234) when
 * tree_theta == 0.  closest/closestd are host outputs (NULL skips). */
int qv_closest(qv_ctx *ctx, int *closest, double *closestd);

/* energy_info (src/diagnostic.f90:259-280) with the context's velocities. */
int qv_energy(qv_ctx *ctx, double *energy);

/* One pass of the loop body of src/run.f90:41-107 restricted to the path:
 * ghostp, construct_tree, pmotion/pmotion_RK3, the candidate search when
 * itime % recon_shots == 0, ghostp, boundary wrap.  Device-resident. */
int qv_step(qv_ctx *ctx, int itime);
/* nsteps steps itime0, itime0+1, ... with the results of calling qv_step for
 * each.  When the point set cannot change and no step needs a host decision
 * (Adams-Bashforth, line_ops 0, tree_theta 0 with velocity BS, LIA or Off, a
 * context stream other than the legacy or per-thread default stream), the
 * steps after the first are replayed from a CUDA graph of one step and the
 * call waits once, at the end; a singularity is then reported after the last
 * step rather than at the step where it occurred.  Otherwise it loops over
 * qv_step.  Not a reference routine: it is the time loop of src/run.f90:36-107
 * run nsteps times between two outputs. */
int qv_steps(qv_ctx *ctx, int itime0, int nsteps);

/* ------------------------------------------------------------- derivatives
 * Hand-written derivatives of the path (no counterpart in the reference, which
 * has no adjoint; they serve gradient-based studies and the stiff solver). */
/* calc_velocity for every active point into a device array u (3n). */
int qv_velocity_device(qv_ctx *ctx, double *u);
/* x_bar = J^T u_bar of calc_velocity (src/timestep.f90:180-309) at the
 * context's positions, through LIA, the direct sum or the tree walk (topology
 * of the current tree frozen) and the ghost gather.  Device pointers (3n). */
int qv_velocity_vjp(qv_ctx *ctx, const double *u_bar, double *x_bar);
/* energy_info (src/diagnostic.f90:259-280) for the context's positions and the
 * device velocities u, with dE/dx (explicit, through s' and the segment
 * lengths) and dE/du, device pointers (3n); energy on the host, its per-point
 * terms summed with compensation (qv_energy sums them in the reference's
 * sequential order). */
int qv_energy_grad(qv_ctx *ctx, const double *u, double *energy, double *x_bar, double *u_bar);
/* One position update of pmotion (src/timestep.f90:48-71: the Adams-Bashforth
 * ladder, rung chosen per point by exact-zero tests of the history) followed by
 * enforce_periodic (src/periodic.f90:188-214), from device arrays x, u, u1, u2,
 * u3 (3n each, n = the context's slot count, its infront marking empty slots)
 * into x_out; the same operations as qv_step's update, so x_out is bitwise what
 * qv_step would store.  Queued on the context's stream. */
int qv_ab_step_device(qv_ctx *ctx, int n, const double *x, const double *u, const double *u1,
                      const double *u2, const double *u3, double *x_out);
/* Its adjoint: given x_out_bar, x_bar = x_out_bar and u_bar, u1_bar, u2_bar,
 * u3_bar = the rung's coefficients times x_out_bar (zero for empty slots);
 * u1..u3 select the rung.  Device pointers (3n each). */
int qv_ab_vjp_device(qv_ctx *ctx, int n, const double *u1, const double *u2, const double *u3,
                     const double *x_out_bar, double *x_bar, double *u_bar, double *u1_bar,
                     double *u2_bar, double *u3_bar);
/* biot_savart_general(_shift) (src/timestep.f90:516-563) at m host points and
 * the exact gradient du_i/dx_k (9 per point, row-major) -- the derivative that
 * velocity_quasip takes by central differences (src/hamiltonian.f90:65-89).
 * grad_images = 0 differentiates the unshifted sum as the reference does. */
int qv_field_velocity(qv_ctx *ctx, int m, const double *pts, int grad_images, double *u,
                      double *dudx);
/* tree_walk_general (src/tree.f90:425-488) at m host points: the Tree arm of
 * mesh_velocity (src/timestep.f90:374-452), the unshifted tree then the
 * boundary's images, on the tree of the last build (built if there is none;
 * needs tree_theta > 0).  Kept as the reference computes it: the leaf term is
 * divided by 4 pi, the far-field term is not, and neither is multiplied by
 * quant_circ; a cell whose centroid lies within epsilon of the point adds
 * nothing.  u: 3m host values; *evals (may be NULL): evaluations. */
int qv_field_velocity_tree(qv_ctx *ctx, int m, const double *pts, double *u, long long *evals);

/* ---------------------------------------------------------------- host side
 * The parts of the reference's driver that feed this path, for a host that
 * runs without the Fortran code (qvort_run) or a test. */
typedef struct qv_run {
  qv_params p;          /* the path's parameters (gpu_precision selects FP64/mixed) */
  int nsteps, shots, pcount, readin_var_file, switch_off_recon;
  char initf[32];
} qv_run;
/* read_run_file (src/cdata.f90:420-807) for the keys of this path; unknown
 * labels are ignored and a value that fails to read ends the file, as there. */
int qv_read_run_file(const char *path, qv_run *out);
/* read_var_file (src/initial.f90:463-496): t, pcount, x, y, z, infront;
 * behind reconstructed as there.  With x == NULL only *n and *t are set. */
int qv_read_var_file(const char *path, int cap, int *n, double *t, double *x, int *infront,
                     int *behind);
/* printf (src/output.f90:116-143): the var%04d.log stream snapshot. */
int qv_write_var_file(const char *path, int n, double t, const double *x, const int *infront,
                      const double *u);
/* The point fields of a restart file (host arrays of at least n slots: 3 per
 * slot for vectors, 1 for links and closest/closestd; NULL skips a field on
 * either side, x/infront/behind are required to write). */
typedef struct qv_restart {
  double *x, *u, *u1, *u2, *u3, *u_li, *u_bs, *gi, *gb, *gii, *gbb, *closestd;
  int *infront, *behind, *closest;
} qv_restart;
/* data_dump (src/output.f90:272-285): ./data/var.dat as gfortran writes it --
 * sequential unformatted records framed by 4-byte length markers: pcount,
 * recon_count, itime, t, f(:) (pcount records of type qvort,
 * src/cdata.f90:20-39, under -fdefault-real-8: 464 bytes each in declaration
 * order with natural alignment), quasi_pcount = 0, part_count = 0.  Fields of
 * qvort outside this path (x_interp, acc, u_mf, f_mf, stretch, curv,
 * closestd_loop, pinned flags, t_recon) are written as zero, u_sup as u and
 * the resolution factor delta as 1.  Files of 2 GiB or more (above ~4.6M
 * slots) are refused with QV_ERR_ARG. */
int qv_write_restart_file(const char *path, int n, int recon_count, int itime, double t,
                          const qv_restart *s);
/* data_restore (src/initial.f90:501-538): *n = pcount, recon_count, itime and
 * t, and, when s and s->x are given, the fields of the first *n <= cap slots.
 * A file whose f(:) record is not pcount * 464 bytes returns QV_ERR_ARG. */
int qv_read_restart_file(const char *path, int cap, int *n, int *recon_count, int *itime,
                         double *t, qv_restart *s);
/* data_dump of the context's state, from its device buffers: positions,
 * velocities (u, u_s_LI, u_s_BS), history, ghosts, links, closest and closestd
 * as the last step left them. */
int qv_dump(qv_ctx *ctx, const char *path, int recon_count, int itime, double t);
/* data_restore into the context: the positions, links, history and closest of
 * the file (as qv_set_state), its pcount in the context; itime, t and
 * recon_count returned.  The run resumes with qv_step(itime + 1): a resumed
 * run is bitwise the run that was never interrupted. */
int qv_restore(qv_ctx *ctx, const char *path, int *recon_count, int *itime, double *t);
/* printf (src/output.f90:116-143) from the context's device buffers: the
 * var%04d.log stream snapshot of the current positions, links and u. */
int qv_write_snapshot(qv_ctx *ctx, const char *path, double t);

/* setup_single_loop / setup_leap_frog (src/initial_loop.f90:11-38, 206-245). */
int qv_setup_loops(const char *initf, int pcount, double delta, double *x, int *infront,
                   int *behind);

/* Block until the context's stream is idle. */
int qv_sync(qv_ctx *ctx);
/* Line operations (replacing `call pinsert` / `call premove`, src/run.f90:59, 72).
 * pinsert (src/line.f90:18-106; delta_adapt and mirror off): points inserted
 * where the distance to the infront ghost exceeds delta, in the reference's
 * slot order, on the stored ghosts (those of the last ghost gather, as after
 * pmotion).  Empty slots are filled first (minloc), then slots are appended:
 * the slot count can grow (qv_point_count).  *inserted may be NULL. */
int qv_pinsert(qv_ctx *ctx, int *inserted);
/* premove (src/line.f90:112-161; phonon emission and recon_info off) with
 * loop_killer (src/reconnection.f90:421-461): the point infront of i goes when
 * |x_i - x_infront(infront(i))| < 0.998 delta; loops left with fewer than 5
 * points are cleared.  *removed (may be NULL) counts both. */
int qv_premove(qv_ctx *ctx, int *removed);
/* precon with recon_type 'original' (src/reconnection.f90:145-254; recon_info
 * and recon_time_info off): reconnects each point whose last candidate search
 * (qv_closest) found a partner closer than delta/2, unless the filaments are
 * near parallel or the line would lengthen; loops left below 5 points are
 * cleared.  Uses the stored ghosts.  *count (may be NULL) = reconnections. */
int qv_precon(qv_ctx *ctx, int *count);
/* Current slot count (pcount), which pinsert can raise, and the links of all
 * slots (1-based, 0 = empty slot; the f(:)%infront, f(:)%behind a host
 * scatters back after insertion or removal). */
int qv_point_count(qv_ctx *ctx, int *n);
int qv_get_links(qv_ctx *ctx, int *infront, int *behind);

/* Instrumentation (no reference counterpart beyond the seg_fault trace flags,
 * src/run.f90:31-166, and eval_counter, src/tree.f90:40).  With profiling on,
 * the phases below are bracketed by CUDA events on the context's stream and
 * their device times accumulate into ms[QV_NPHASES]. */
/* ghosts, tree build, local term, non-local sum, update, search, wrap, two
 * parts of the tree build (the level-synchronous construction and the
 * moments), the line operations (pinsert, premove), and inside the non-local
 * sum the mixed Barnes-Hut walk's kernel alone */
#define QV_NPHASES 11
int qv_profile(qv_ctx *ctx, int enable);
int qv_phase_times(qv_ctx *ctx, double *ms, int reset);
/* Kernel launches issued by this context so far, and the leaf / far-field
 * evaluations of the last tree walk. */
int qv_counters(qv_ctx *ctx, long long *launches, long long *leaf_evals, long long *far_evals);
/* Measured FP32 FMA throughput of the current device (TFLOP/s), the
 * denominator of the FP32-pipe roofline. */
int qv_probe_fp32(void *stream, double *tflops);

/* Test hook, no counterpart in the reference: enable != 0 makes every
 * source-tile wait of the direct-sum kernels report that it ran out, without
 * waiting, so the bounded-wait error path (drain the copies in flight, flag
 * the status word, return QV_ERR_CUDA) can be exercised while every copy
 * still lands; 0 restores normal waits.  Process-wide. */
int qv_test_stage_timeout(int enable);

/* Test hook, no counterpart in the reference: how the tree's root centroid is
 * taken.  mode -1 (the default): trees of at least 32768 slots start the
 * build and the walk from a bounded estimate of the root centroid while its
 * exact sequential sum runs alongside, and fix up the root tests the bound
 * leaves undecided (results are those of the exact centroid); 0: always wait
 * for the exact sum; 1: always start from the estimate.  bound_scale >= 1
 * widens the estimate's bound, so that a test can make root tests undecided
 * and exercise the fix-up.  Process-wide. */
int qv_test_root_speculation(int mode, double bound_scale);

/* Test hook, no counterpart in the reference: when a mixed-precision Tree
 * build takes the root children's long circ and Cij sums off the path to the
 * walk.  mode -1 (the default): builds of at least 65536 slots pack the
 * children of more than 512 points late, and the walk adds their far-field
 * terms after its launch (results within the mixed walk's rounding of the
 * other path, same evaluation counts); 0: never; 1: always.  Process-wide. */
int qv_test_late_level1(int mode);
/* The number of root tests the last estimate-started build left undecided
 * (see qv_test_root_speculation; 0 when the build waited for the exact sum). */
int qv_root_undecided(qv_ctx *ctx, int *count);

/* Non-local direct Biot-Savart velocity without any device allocation.
 * No counterpart in the reference: it exists for hosts that cannot call
 * cudaMalloc/cudaFree on their hot path -- drivers that reserve their whole
 * device memory budget up front, codes embedded in a framework that owns the
 * allocator, loops that cannot afford the device synchronisation of
 * cudaMalloc/cudaFree.  It computes what qv_velocity returns in u_bs for
 * velocity BS (the direct sum with the periodic images of p->boundary, in
 * p->precision) from device pointers x (3n), infront, behind (n) into the
 * device array u_bs (3n), on stream (NULL = legacy default stream), and
 * returns when the result is complete.  Temporaries live in one file-scope
 * device array sized for QV_NOALLOC_MAX_POINTS slots (about 9 MB, held by
 * every GPU that loads the library until exit); n above that returns
 * QV_ERR_NOALLOC_LIMIT.  The first call on a device looks up that array's
 * address (cudaGetSymbolAddress) and should come before any stream capture;
 * the address is kept for the life of the process, so the library must not be
 * used on a device across a cudaDeviceReset.  Each call waits for its stream
 * before it returns.  All calls share the array: calls that overlap on the GPU
 * race and must be serialised by the caller. */
#define QV_NOALLOC_MAX_POINTS 16384
int qv_velocity_direct_noalloc(const qv_params *p, int n, const double *x, const int *infront,
                               const int *behind, double *u_bs, void *stream);

/* ---------------------------------------------------------------- batches
 * Many independent systems advanced together (no counterpart in the
 * reference, which runs one system per process; each system is what one run
 * of src/run.f90's loop would hold).  nsys systems occupy consecutive slot
 * ranges [offsets[s], offsets[s+1]) of one point array; method[s] is
 * QV_VEL_BS (direct sum) or QV_VEL_TREE (Barnes-Hut with p->tree_theta), dt[s]
 * the system's time step.  Every system has open boundaries and its own box of
 * side p->box_size centred on the origin of its coordinates; p->boundary must
 * be QV_BC_OPEN and p->precision QV_PREC_MIXED (else QV_ERR_UNSUPPORTED).
 * stream: as for qv_create; graph capture needs a stream other than the
 * legacy default stream (NULL gives a private one). */
typedef struct qv_batch qv_batch;
int qv_batch_create(const qv_params *p, int nsys, const int *offsets, const int *method,
                    const double *dt, void *stream, qv_batch **out);
void qv_batch_destroy(qv_batch *b);
const char *qv_batch_last_error(qv_batch *b);
/* Positions x (3 per slot) and each system's own 1-based links (1..n_s; no
 * empty slots); clears the Adams-Bashforth history. */
int qv_batch_set_points(qv_batch *b, const double *x, const int *infront, const int *behind);
/* calc_velocity of every system at the current positions (u: 3 per slot,
 * host, may be NULL); positions and history unchanged. */
int qv_batch_velocity(qv_batch *b, double *u);
/* nsteps steps of velocity + pmotion for every system: one CUDA graph launch
 * per step when capture succeeds, otherwise the same launches issued
 * directly.  Returns when all steps are done. */
int qv_batch_step(qv_batch *b, int nsteps);
int qv_batch_get_points(qv_batch *b, double *x, double *u);
/* Times the persistent work kernel under each launch shape and keeps the
 * fastest; best_cfg = {warps per block, blocks per SM, order (1 = largest
 * items first)}.  Results are identical under every shape. */
int qv_batch_tune(qv_batch *b, int reps, int *best_cfg, float *best_ms);
int qv_batch_set_config(qv_batch *b, int warps_per_block, int blocks_per_sm, int order);
/* evals[0..1] = leaf and far-field evaluations of the last step; graph_used;
 * config[0..7] = warps per block, blocks per SM, order, walk stack entries,
 * work items, tree systems, forest depth, launches issued so far. */
int qv_batch_stats(qv_batch *b, long long *evals, int *graph_used, int *config);

#ifdef __cplusplus
}
#endif
#endif
