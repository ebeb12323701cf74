! mhd_gpu_bind.f90 -- ISO_C_BINDING interfaces to libmhd_gpu.so (include/mhd_gpu.h).
!
! A Fortran driver (drive.f90 of YueWu2002/PP-ES-DG-MHD) uses this module in place of calling
! DG_solver_m's procedures directly.  Arrays keep the reference's explicit-shape, column-major
! layouts; handles are type(c_ptr).  Every function returns integer(c_int): 0 = OK, > 0 = solver
! flag bits (MHD_FLAG_*), < 0 = API error.
!
! The module declares every function, constant and struct of include/mhd_gpu.h, in the header's
! order; a CPU test (tests/test_fortran_binding.py) parses both files and checks that the function
! lists, argument counts, pass-by-value attributes and struct fields agree.  No Fortran compiler
! exists on the machine that produced this repository, so the module itself was not compiled there.
!
! Pointer arguments the header allows to be NULL (neg_avg, num_negcell, tot_ent, dt_lim, ...) are
! declared here as ordinary by-reference arguments: a Fortran caller always passes a variable.
module mhd_gpu_bind
  use, intrinsic :: iso_c_binding
  implicit none

  ! status codes
  integer(c_int), parameter :: MHD_OK = 0
  integer(c_int), parameter :: MHD_FLAG_NEG_AVG = 1, MHD_FLAG_PP_RELIMIT = 2
  integer(c_int), parameter :: MHD_FLAG_DT_COLLAPSE = 4, MHD_FLAG_INIT_NEG_AVG = 8
  integer(c_int), parameter :: MHD_FLAG_DEVICE_WAIT = 16
  integer(c_int), parameter :: MHD_ERR_INVALID = -1, MHD_ERR_UNSUPPORTED = -2, MHD_ERR_CUDA = -3
  integer(c_int), parameter :: MHD_ERR_NO_DEVICE = -4, MHD_ERR_STATE = -5
  ! boundary-condition kinds (replace the BC_handle procedure pointer, drive.f90:25)
  integer(c_int), parameter :: MHD_BC_PERIODIC = 0, MHD_BC_EXTRAPOLATE = 1
  integer(c_int), parameter :: MHD_BC_FIXED = 2, MHD_BC_XEXTRAP_YPER = 3
  integer(c_int), parameter :: MHD_BC_CLOUD_SHOCK = 4, MHD_BC_JET = 5
  ! set-ups evaluated on the device (mhd_gpu_init_problem)
  integer(c_int), parameter :: MHD_IC_OT2PI = 0, MHD_IC_OT_UNIT = 1, MHD_IC_VORTEX = 2
  integer(c_int), parameter :: MHD_IC_BLAST = 3, MHD_IC_ROTOR = 4, MHD_IC_ALFVEN = 5
  integer(c_int), parameter :: MHD_IC_CLOUD_SHOCK = 6, MHD_IC_JET = 7
  ! driver log record kinds
  integer(c_int), parameter :: MHD_LOG_STAGE = 1, MHD_LOG_STEP = 2

  type, bind(C) :: mhd_gpu_status
    real(c_double) :: t, dt, dt_lim, tot_ent
    integer(c_long_long) :: steps, retries, num_negcell_total
    integer(c_int) :: num_negcell_last, done, flags, pad_
  end type mhd_gpu_status

  type, bind(C) :: mhd_log_entry
    integer(c_long_long) :: seq, step
    integer(c_int) :: kind, stage, try_num, num_negcell, neg_avg, flags
    real(c_double) :: t, dt, dt_lim, tot_ent, rho_min, p_min
    real(c_double) :: total(8)
  end type mhd_log_entry

  type, bind(C) :: mhd_request
    integer(c_long_long) :: id
    integer(c_int) :: nx, ny, p, rknstg
    real(c_double) :: left, right, bottom, top, gamma
    integer(c_int) :: bc_kind, pad_
    real(c_double) :: bc_state8(8)
    real(c_double) :: final_T, cfl
    integer(c_int) :: use_oedg, use_ldf, ent_offset, pad2_
    real(c_double) :: arrival
    type(c_ptr) :: u0, u_avg_out
  end type mhd_request

  type, bind(C) :: mhd_request_result
    integer(c_long_long) :: id
    real(c_double) :: arrival, admitted, finished
    real(c_double) :: t
    integer(c_long_long) :: steps, retries
    integer(c_int) :: done, flags, error, pad_
  end type mhd_request_result

  type, bind(C) :: mhd_server_stats
    integer(c_long_long) :: rounds
    integer(c_long_long) :: admitted, retired
    integer(c_long_long) :: graph_captures
    real(c_double) :: admit_s, launch_s, wait_s, retire_s, idle_s
  end type mhd_server_stats

  interface
    ! ---- life cycle ----
    integer(c_int) function mhd_gpu_create(nx, ny, px, py, rknstg, left, right, bottom, top, &
                                           gamma, bc_kind, bc_state8, h) bind(C, name="mhd_gpu_create")
      import :: c_int, c_double, c_ptr
      integer(c_int), value :: nx, ny, px, py, rknstg
      real(c_double), value :: left, right, bottom, top, gamma
      integer(c_int), value :: bc_kind
      real(c_double), intent(in) :: bc_state8(*)
      type(c_ptr), intent(out) :: h
    end function

    integer(c_int) function mhd_gpu_destroy(h) bind(C, name="mhd_gpu_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function

    integer(c_int) function mhd_gpu_set_stream(h, cuda_stream) bind(C, name="mhd_gpu_set_stream")
      import :: c_int, c_ptr
      type(c_ptr), value :: h, cuda_stream
    end function

    integer(c_int) function mhd_gpu_device_bytes(h, bytes) bind(C, name="mhd_gpu_device_bytes")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: h
      integer(c_size_t), intent(out) :: bytes
    end function

    integer(c_int) function mhd_gpu_synchronize(h) bind(C, name="mhd_gpu_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function

    ! returns a C string (const char*); convert with c_f_pointer on the caller's side
    type(c_ptr) function mhd_gpu_status_string(code) bind(C, name="mhd_gpu_status_string")
      import :: c_int, c_ptr
      integer(c_int), value :: code
    end function

    ! ---- geometry and tables ----
    integer(c_int) function mhd_gpu_nodes(h, xx, yy) bind(C, name="mhd_gpu_nodes")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: xx(*), yy(*)
    end function

    integer(c_int) function mhd_gpu_gll_tables(p, x, w, m, minv, d, pmn, pnm) bind(C, name="mhd_gpu_gll_tables")
      import :: c_int, c_double
      integer(c_int), value :: p
      real(c_double), intent(out) :: x(*), w(*), m(*), minv(*), d(*), pmn(*), pnm(*)
    end function

    integer(c_int) function mhd_gpu_ldf_operator(p, hx, hy, a) bind(C, name="mhd_gpu_ldf_operator")
      import :: c_int, c_double
      integer(c_int), value :: p
      real(c_double), value :: hx, hy
      real(c_double), intent(out) :: a(*)
    end function

    ! ---- state transfer (Fortran layouts) ----
    integer(c_int) function mhd_gpu_upload_state(h, slot, u) bind(C, name="mhd_gpu_upload_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: slot
      real(c_double), intent(in) :: u(*)
    end function

    integer(c_int) function mhd_gpu_download_state(h, slot, u) bind(C, name="mhd_gpu_download_state")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: slot
      real(c_double), intent(out) :: u(*)
    end function

    integer(c_int) function mhd_gpu_upload_ut(h, stage, ut) bind(C, name="mhd_gpu_upload_ut")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: stage
      real(c_double), intent(in) :: ut(*)
    end function

    integer(c_int) function mhd_gpu_download_ut(h, stage, ut) bind(C, name="mhd_gpu_download_ut")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: stage
      real(c_double), intent(out) :: ut(*)
    end function

    integer(c_int) function mhd_gpu_download_avg(h, u_avg) bind(C, name="mhd_gpu_download_avg")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: u_avg(*)
    end function

    ! buffer_var(nx+1, ny, 8) real(c_float), var_min(8), var_max(8): the arrays of
    ! save_tecbin_finite_volume (io.f90:75-86)
    integer(c_int) function mhd_gpu_download_avg_primitive(h, buffer_var, var_min, var_max) &
        bind(C, name="mhd_gpu_download_avg_primitive")
      import :: c_int, c_ptr, c_double, c_float
      type(c_ptr), value :: h
      real(c_float), intent(out) :: buffer_var(*)
      real(c_double), intent(out) :: var_min(*), var_max(*)
    end function

    ! ---- initial state on the device ----
    integer(c_int) function mhd_gpu_init_problem(h, problem, params, nparams) bind(C, name="mhd_gpu_init_problem")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: problem
      real(c_double), intent(in) :: params(*)
      integer(c_int), value :: nparams
    end function

    ! ---- the reference's per-call interface ----
    integer(c_int) function mhd_gpu_apply_bc(h, slot) bind(C, name="mhd_gpu_apply_bc")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: slot
    end function

    integer(c_int) function mhd_gpu_post_process(h, slot, apply_oedg, apply_ldf, oedg_dt, &
                                                 ent_offset, comput_ent, neg_avg, num_negcell, &
                                                 tot_ent) bind(C, name="mhd_gpu_post_process")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: slot, apply_oedg, apply_ldf
      real(c_double), value :: oedg_dt
      integer(c_int), value :: ent_offset, comput_ent
      integer(c_int), intent(out) :: neg_avg, num_negcell
      real(c_double), intent(out) :: tot_ent
    end function

    integer(c_int) function mhd_gpu_semidiscretize(h, ut_stage, slot, dt_lim) &
        bind(C, name="mhd_gpu_semidiscretize")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: ut_stage, slot
      real(c_double), intent(out) :: dt_lim
    end function

    integer(c_int) function mhd_gpu_rk_combine(h, stage, dt) bind(C, name="mhd_gpu_rk_combine")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      integer(c_int), value :: stage
      real(c_double), value :: dt
    end function

    integer(c_int) function mhd_gpu_rk_accept(h) bind(C, name="mhd_gpu_rk_accept")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function

    ! ---- device-resident solve_execute ----
    integer(c_int) function mhd_gpu_solve_begin(h, final_T, cfl, use_oedg, use_ldf, ent_offset, &
                                                tot_ent, dt_lim) bind(C, name="mhd_gpu_solve_begin")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), value :: final_T, cfl
      integer(c_int), value :: use_oedg, use_ldf, ent_offset
      real(c_double), intent(out) :: tot_ent, dt_lim
    end function

    integer(c_int) function mhd_gpu_step(h, st) bind(C, name="mhd_gpu_step")
      import :: c_int, c_ptr, mhd_gpu_status
      type(c_ptr), value :: h
      type(mhd_gpu_status), intent(out) :: st
    end function

    integer(c_int) function mhd_gpu_advance(h, max_steps, check_every, st) bind(C, name="mhd_gpu_advance")
      import :: c_int, c_ptr, c_long_long, mhd_gpu_status
      type(c_ptr), value :: h
      integer(c_long_long), value :: max_steps
      integer(c_int), value :: check_every
      type(mhd_gpu_status), intent(out) :: st
    end function

    integer(c_int) function mhd_gpu_get_status(h, st) bind(C, name="mhd_gpu_get_status")
      import :: c_int, c_ptr, mhd_gpu_status
      type(c_ptr), value :: h
      type(mhd_gpu_status), intent(out) :: st
    end function

    ! ---- driver log (the stage prints and entropy log of drive.f90:74,285-294,314) ----
    integer(c_int) function mhd_gpu_set_log(h, capacity, diagnostics) bind(C, name="mhd_gpu_set_log")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: capacity, diagnostics
    end function

    integer(c_int) function mhd_gpu_read_log(h, out, cap, n, dropped) bind(C, name="mhd_gpu_read_log")
      import :: c_int, c_ptr, c_long_long, mhd_log_entry
      type(c_ptr), value :: h
      type(mhd_log_entry), intent(out) :: out(*)
      integer(c_int), value :: cap
      integer(c_int), intent(out) :: n
      integer(c_long_long), intent(out) :: dropped
    end function

    integer(c_int) function mhd_gpu_state_device_ptr(h, slot, dptr) bind(C, name="mhd_gpu_state_device_ptr")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: slot
      type(c_ptr), intent(out) :: dptr
    end function

    integer(c_int) function mhd_gpu_step_graph_kernels(h, n) bind(C, name="mhd_gpu_step_graph_kernels")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
      integer(c_int), intent(out) :: n
    end function

    ! ---- many instances advanced together (no reference counterpart) ----
    integer(c_int) function mhd_batch_create(b) bind(C, name="mhd_batch_create")
      import :: c_int, c_ptr
      type(c_ptr), intent(out) :: b
    end function

    integer(c_int) function mhd_batch_destroy(b) bind(C, name="mhd_batch_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: b
    end function

    integer(c_int) function mhd_batch_add(b, h) bind(C, name="mhd_batch_add")
      import :: c_int, c_ptr
      type(c_ptr), value :: b, h
    end function

    integer(c_int) function mhd_batch_remove(b, h) bind(C, name="mhd_batch_remove")
      import :: c_int, c_ptr
      type(c_ptr), value :: b, h
    end function

    integer(c_int) function mhd_batch_size(b, n) bind(C, name="mhd_batch_size")
      import :: c_int, c_ptr
      type(c_ptr), value :: b
      integer(c_int), intent(out) :: n
    end function

    integer(c_int) function mhd_batch_advance(b, tries, n_active) bind(C, name="mhd_batch_advance")
      import :: c_int, c_ptr
      type(c_ptr), value :: b
      integer(c_int), value :: tries
      integer(c_int), intent(out) :: n_active
    end function

    integer(c_int) function mhd_batch_launch(b, tries) bind(C, name="mhd_batch_launch")
      import :: c_int, c_ptr
      type(c_ptr), value :: b
      integer(c_int), value :: tries
    end function

    integer(c_int) function mhd_batch_wait(b, n_active) bind(C, name="mhd_batch_wait")
      import :: c_int, c_ptr
      type(c_ptr), value :: b
      integer(c_int), intent(out) :: n_active
    end function

    integer(c_int) function mhd_batch_member_status(b, h, st) bind(C, name="mhd_batch_member_status")
      import :: c_int, c_ptr, mhd_gpu_status
      type(c_ptr), value :: b, h
      type(mhd_gpu_status), intent(out) :: st
    end function

    ! ---- serving (no reference counterpart) ----
    integer(c_int) function mhd_gpu_footprint(nx, ny, p, rknstg, bytes) bind(C, name="mhd_gpu_footprint")
      import :: c_int, c_size_t
      integer(c_int), value :: nx, ny, p, rknstg
      integer(c_size_t), intent(out) :: bytes
    end function

    integer(c_int) function mhd_server_create(hbm_budget_bytes, max_active, tries_per_round, batched, s) &
        bind(C, name="mhd_server_create")
      import :: c_int, c_ptr, c_size_t
      integer(c_size_t), value :: hbm_budget_bytes
      integer(c_int), value :: max_active, tries_per_round, batched
      type(c_ptr), intent(out) :: s
    end function

    integer(c_int) function mhd_server_submit(s, r) bind(C, name="mhd_server_submit")
      import :: c_int, c_ptr, mhd_request
      type(c_ptr), value :: s
      type(mhd_request), intent(in) :: r
    end function

    integer(c_int) function mhd_server_run(s, max_seconds) bind(C, name="mhd_server_run")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: s
      real(c_double), value :: max_seconds
    end function

    integer(c_int) function mhd_server_pending(s, queued, active, used_bytes) bind(C, name="mhd_server_pending")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: s
      integer(c_int), intent(out) :: queued, active
      integer(c_size_t), intent(out) :: used_bytes
    end function

    integer(c_int) function mhd_server_results(s, out, cap, n) bind(C, name="mhd_server_results")
      import :: c_int, c_ptr, mhd_request_result
      type(c_ptr), value :: s
      type(mhd_request_result), intent(out) :: out(*)
      integer(c_int), value :: cap
      integer(c_int), intent(out) :: n
    end function

    integer(c_int) function mhd_server_get_stats(s, out) bind(C, name="mhd_server_get_stats")
      import :: c_int, c_ptr, mhd_server_stats
      type(c_ptr), value :: s
      type(mhd_server_stats), intent(out) :: out
    end function

    integer(c_int) function mhd_server_destroy(s) bind(C, name="mhd_server_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: s
    end function

    ! ---- allocation-free residual (no reference counterpart) ----
    ! u, ut: device addresses (type(c_ptr)) of caller-owned arrays; stream: a cudaStream_t
    integer(c_int) function mhd_gpu_semidiscretize_noalloc(p, nx, ny, hx, hy, gamma, u, ut, dt_lim, stream) &
        bind(C, name="mhd_gpu_semidiscretize_noalloc")
      import :: c_int, c_ptr, c_double
      integer(c_int), value :: p, nx, ny
      real(c_double), value :: hx, hy, gamma
      type(c_ptr), value :: u, ut
      real(c_double), intent(out) :: dt_lim
      type(c_ptr), value :: stream
    end function
  end interface
end module mhd_gpu_bind
