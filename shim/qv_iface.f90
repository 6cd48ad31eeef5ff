!> ISO_C_BINDING interface to the B200 velocity-and-timestep path
!> (include/qv.h).  A maintainer adds this module to the reference's
!> src/Makefile and links libqvort_b200.so.  Each wrapper below names the
!> reference routine (file:line) whose call it replaces in src/run.f90 or
!> src/timestep.f90.
!>
!> f(:) is not bind(C), so every call gathers the fields it needs into
!> contiguous arrays and scatters results back; it never aliases the AoS.
!> All calls are made from the serial region (never inside !$omp parallel).
module qv_iface
  use, intrinsic :: iso_c_binding
  use cdata
  implicit none
  private
  public :: qv_gpu_init, qv_gpu_step, qv_gpu_velocity, qv_gpu_pclose, qv_gpu_finish

  integer(c_int), parameter :: QV_BC_OPEN = 0, QV_BC_PERIODIC = 1, QV_BC_OPENX = 2, &
                               QV_BC_OPENXY = 3
  integer(c_int), parameter :: QV_VEL_OFF = 0, QV_VEL_LIA = 1, QV_VEL_BS = 2, QV_VEL_TREE = 3

  type, bind(C) :: qv_params_t
    real(c_double) :: quant_circ, corea, box_size, delta, dt, tree_theta
    integer(c_int) :: boundary, velocity, deriv_order, tree_extra_correction
    integer(c_int) :: fixed_lia_beta, precision, runge_kutta, recon_shots
    integer(c_int) :: line_ops
  end type

  ! the per-step exchange of qv_set_state / qv_get_state (host arrays by address)
  type, bind(C) :: qv_state_t
    type(c_ptr) :: x, u, u1, u2, u3, infront, behind, closest, closestd
  end type

  interface
    integer(c_int) function qv_default_params(p) bind(C, name='qv_default_params')
      import :: qv_params_t
      type(qv_params_t), intent(out) :: p
    end function
    integer(c_int) function qv_create(p, stream, ctx) bind(C, name='qv_create')
      import :: qv_params_t, c_ptr
      type(qv_params_t), intent(in) :: p
      type(c_ptr), value :: stream
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function qv_destroy(ctx) bind(C, name='qv_destroy')
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function qv_set_points(ctx, n, x, infront, behind) bind(C, name='qv_set_points')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      real(c_double), intent(in) :: x(3, *)
      integer(c_int), intent(in) :: infront(*), behind(*)
    end function
    integer(c_int) function qv_set_history(ctx, u1, u2, u3) bind(C, name='qv_set_history')
      import :: c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(in) :: u1(3, *), u2(3, *), u3(3, *)
    end function
    integer(c_int) function qv_get_history(ctx, u1, u2, u3) bind(C, name='qv_get_history')
      import :: c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: u1(3, *), u2(3, *), u3(3, *)
    end function
    integer(c_int) function qv_set_closest(ctx, closest) bind(C, name='qv_set_closest')
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), intent(in) :: closest(*)
    end function
    integer(c_int) function qv_get_points(ctx, x, u) bind(C, name='qv_get_points')
      import :: c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: x(3, *), u(3, *)
    end function
    integer(c_int) function qv_get_closest(ctx, closest, closestd) bind(C, name='qv_get_closest')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: closest(*)
      real(c_double), intent(out) :: closestd(*)
    end function
    integer(c_int) function qv_step(ctx, itime) bind(C, name='qv_step')
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
      integer(c_int), value :: itime
    end function
    integer(c_int) function qv_velocity(ctx, u, u_li, u_bs, eval_count) bind(C, name='qv_velocity')
      import :: c_ptr, c_double, c_long_long
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: u(3, *), u_li(3, *), u_bs(3, *)
      integer(c_long_long), intent(out) :: eval_count
    end function
    integer(c_int) function qv_closest(ctx, closest, closestd) bind(C, name='qv_closest')
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), intent(out) :: closest(*)
      real(c_double), intent(out) :: closestd(*)
    end function
    type(c_ptr) function qv_last_error(ctx) bind(C, name='qv_last_error')
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function qv_set_state(ctx, n, s) bind(C, name='qv_set_state')
      import :: c_ptr, c_int, qv_state_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: n
      type(qv_state_t), intent(in) :: s
    end function
    integer(c_int) function qv_get_state(ctx, cap, s, n) bind(C, name='qv_get_state')
      import :: c_ptr, c_int, qv_state_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: cap
      type(qv_state_t), intent(in) :: s
      integer(c_int), intent(out) :: n
    end function
    integer(c_int) function qv_step_exchange(ctx, itime, n, sin, cap, sout, nout) &
        bind(C, name='qv_step_exchange')
      import :: c_ptr, c_int, qv_state_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: itime, n, cap
      type(qv_state_t), intent(in) :: sin, sout
      integer(c_int), intent(out) :: nout
    end function
  end interface

  type(c_ptr), save :: ctx = c_null_ptr
  real(c_double), allocatable, target, save :: xs(:,:), us(:,:), h1(:,:), h2(:,:), h3(:,:)
  real(c_double), allocatable, target, save :: cds(:), uli(:,:), ubs(:,:)
  integer(c_int), allocatable, target, save :: infs(:), behs(:), cls(:)

contains

  subroutine check(rc, where)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: where
    character(kind=c_char), pointer :: msg(:)
    character(len=256) :: text
    integer :: k
    if (rc == 0) return
    text = ' '
    call c_f_pointer(qv_last_error(ctx), msg, [256])
    do k = 1, 256
      if (msg(k) == c_null_char) exit
      text(k:k) = msg(k)
    end do
    call fatal_error(where, trim(text))   ! cdata.f90:955-970
  end subroutine

  !> build the parameter block from the run.in values read by read_run_file
  subroutine fill_params(p)
    type(qv_params_t), intent(out) :: p
    integer(c_int) :: rc
    rc = qv_default_params(p)
    p%quant_circ = quant_circ ; p%corea = corea ; p%box_size = box_size
    p%delta = delta ; p%dt = dt ; p%tree_theta = tree_theta
    select case (boundary)
      case ('periodic') ; p%boundary = QV_BC_PERIODIC
      case ('openx') ; p%boundary = QV_BC_OPENX
      case ('openxy') ; p%boundary = QV_BC_OPENXY
      case ('open') ; p%boundary = QV_BC_OPEN
      case default ; p%boundary = -1     ! rejected by qv_create
    end select
    select case (velocity)
      case ('Off') ; p%velocity = QV_VEL_OFF
      case ('LIA') ; p%velocity = QV_VEL_LIA
      case ('BS') ; p%velocity = QV_VEL_BS
      case ('Tree') ; p%velocity = QV_VEL_TREE
      case default ; p%velocity = -1
    end select
    p%deriv_order = 2
    if (deriv_order == 'fourth') p%deriv_order = 4
    p%tree_extra_correction = merge(1, 0, tree_extra_correction)
    p%fixed_lia_beta = merge(1, 0, fixed_LIA_beta)
    p%precision = 1                      ! mixed; 0 for FP64 throughout
    p%runge_kutta = merge(1, 0, runge_kutta)
    p%recon_shots = recon_shots
  end subroutine

  subroutine qv_gpu_init()
    type(qv_params_t) :: p
    call fill_params(p)
    call check(qv_create(p, c_null_ptr, ctx), 'qv_iface:qv_create')
  end subroutine

  subroutine gather()
    call gather_arrays()
    call check(qv_set_state(ctx, int(size(f), c_int), state()), 'qv_iface:qv_set_state')
  end subroutine

  subroutine gather_arrays()
    integer :: n
    n = size(f)
    if (allocated(xs)) then
      if (size(xs, 2) /= n) deallocate(xs, us, h1, h2, h3, cds, uli, ubs, infs, behs, cls)
    end if
    if (.not. allocated(xs)) allocate(xs(3,n), us(3,n), h1(3,n), h2(3,n), h3(3,n), cds(n), &
                                      uli(3,n), ubs(3,n), infs(n), behs(n), cls(n))
    xs(1,:) = f(:)%x(1) ; xs(2,:) = f(:)%x(2) ; xs(3,:) = f(:)%x(3)
    h1(1,:) = f(:)%u1(1) ; h1(2,:) = f(:)%u1(2) ; h1(3,:) = f(:)%u1(3)
    h2(1,:) = f(:)%u2(1) ; h2(2,:) = f(:)%u2(2) ; h2(3,:) = f(:)%u2(3)
    h3(1,:) = f(:)%u3(1) ; h3(2,:) = f(:)%u3(2) ; h3(3,:) = f(:)%u3(3)
    infs = f(:)%infront ; behs = f(:)%behind ; cls = f(:)%closest
  end subroutine

  function state() result(s)
    type(qv_state_t) :: s
    s%x = c_loc(xs) ; s%u = c_loc(us) ; s%u1 = c_loc(h1) ; s%u2 = c_loc(h2) ; s%u3 = c_loc(h3)
    s%infront = c_loc(infs) ; s%behind = c_loc(behs) ; s%closest = c_loc(cls)
    s%closestd = c_loc(cds)
  end function

  !> the slot count does not change here (line operations stay on the host)
  subroutine scatter()
    integer(c_int) :: n
    call check(qv_get_state(ctx, int(size(xs, 2), c_int), state(), n), 'qv_iface:qv_get_state')
    call scatter_arrays()
  end subroutine

  subroutine scatter_arrays()
    f(:)%x(1) = xs(1,:) ; f(:)%x(2) = xs(2,:) ; f(:)%x(3) = xs(3,:)
    f(:)%u(1) = us(1,:) ; f(:)%u(2) = us(2,:) ; f(:)%u(3) = us(3,:)
    f(:)%u1(1) = h1(1,:) ; f(:)%u1(2) = h1(2,:) ; f(:)%u1(3) = h1(3,:)
    f(:)%u2(1) = h2(1,:) ; f(:)%u2(2) = h2(2,:) ; f(:)%u2(3) = h2(3,:)
    f(:)%u3(1) = h3(1,:) ; f(:)%u3(2) = h3(2,:) ; f(:)%u3(3) = h3(3,:)
    f(:)%closest = cls ; f(:)%closestd = cds
  end subroutine

  !> replaces ghostp + construct_tree + pmotion|pmotion_RK3 + pclose_tree|pclose
  !> + ghostp + enforce_periodic of src/run.f90:41-84.  The parameters leave
  !> line_ops at 0, so pinsert, precon and premove stay with the host, called
  !> in the reference's order (pinsert after this step's update; precon and
  !> premove after the candidate search, on recon_shots steps)
  subroutine qv_gpu_step(it)
    integer, intent(in) :: it
    integer(c_int) :: n
    call gather_arrays()
    ! set_state + step + get_state in one call, the copies overlapping the step
    call check(qv_step_exchange(ctx, int(it, c_int), int(size(f), c_int), state(), &
                                int(size(xs, 2), c_int), state(), n), 'qv_iface:qv_step_exchange')
    call scatter_arrays()
  end subroutine

  !> replaces the first loop of pmotion (src/timestep.f90:41-47): f(:)%u,
  !> f(:)%u_s_LI, f(:)%u_s_BS for every active point
  subroutine qv_gpu_velocity()
    integer(c_long_long) :: ev
    call gather()
    call check(qv_velocity(ctx, us, uli, ubs, ev), 'qv_iface:qv_velocity')
    f(:)%u(1) = us(1,:) ; f(:)%u(2) = us(2,:) ; f(:)%u(3) = us(3,:)
    f(:)%u_s_LI(1) = uli(1,:) ; f(:)%u_s_LI(2) = uli(2,:) ; f(:)%u_s_LI(3) = uli(3,:)
    f(:)%u_s_BS(1) = ubs(1,:) ; f(:)%u_s_BS(2) = ubs(2,:) ; f(:)%u_s_BS(3) = ubs(3,:)
  end subroutine

  !> replaces pclose_tree / pclose (src/tree.f90:219-234, src/line.f90:205-234)
  subroutine qv_gpu_pclose()
    call check(qv_closest(ctx, cls, cds), 'qv_iface:qv_closest')
    f(:)%closest = cls ; f(:)%closestd = cds
  end subroutine

  subroutine qv_gpu_finish()
    integer(c_int) :: rc
    if (c_associated(ctx)) rc = qv_destroy(ctx)
    ctx = c_null_ptr
  end subroutine
end module
