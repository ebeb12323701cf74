! mhd_gpu_bind.f90 -- ISO_C_BINDING interfaces to libmhd_gpu.so (include/mhd_gpu.h).
!
! A Fortran driver (drive.f90 of YueWu2002/PP-ES-DG-MHD) uses this module in place of calling
! DG_solver_m's procedures directly.  Arrays keep the reference's explicit-shape, column-major
! layouts; handles are type(c_ptr).  Every function returns integer(c_int): 0 = OK, > 0 = solver
! flag bits (MHD_FLAG_*), < 0 = API error.
!
! Not compiled on the machine that produced this repository (no Fortran compiler there); the
! declarations mirror include/mhd_gpu.h one to one.
module mhd_gpu_bind
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: MHD_OK = 0
  integer(c_int), parameter :: MHD_FLAG_NEG_AVG = 1, MHD_FLAG_PP_RELIMIT = 2
  integer(c_int), parameter :: MHD_FLAG_DT_COLLAPSE = 4, MHD_FLAG_INIT_NEG_AVG = 8
  integer(c_int), parameter :: MHD_BC_PERIODIC = 0, MHD_BC_EXTRAPOLATE = 1
  integer(c_int), parameter :: MHD_BC_FIXED = 2, MHD_BC_XEXTRAP_YPER = 3

  type, bind(C) :: mhd_gpu_status
    real(c_double) :: t, dt, dt_lim, tot_ent
    integer(c_long_long) :: steps, retries, num_negcell_total
    integer(c_int) :: num_negcell_last, done, flags, pad_
  end type mhd_gpu_status

  interface
    integer(c_int) function mhd_gpu_create(nx, ny, px, py, rknstg, left, right, bottom, top, &
                                           gamma, bc_kind, bc_state8, h) bind(C, name="mhd_gpu_create")
      import :: c_int, c_double, c_ptr
      integer(c_int), value :: nx, ny, px, py, rknstg, bc_kind
      real(c_double), value :: left, right, bottom, top, gamma
      real(c_double), intent(in) :: bc_state8(*)
      type(c_ptr), intent(out) :: h
    end function

    integer(c_int) function mhd_gpu_destroy(h) bind(C, name="mhd_gpu_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function

    integer(c_int) function mhd_gpu_nodes(h, xx, yy) bind(C, name="mhd_gpu_nodes")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: xx(*), yy(*)
    end function

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

    integer(c_int) function mhd_gpu_download_avg(h, u_avg) bind(C, name="mhd_gpu_download_avg")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(out) :: u_avg(*)
    end function

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
      integer(c_int), value :: slot, apply_oedg, apply_ldf, ent_offset, comput_ent
      real(c_double), value :: oedg_dt
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

    integer(c_int) function mhd_batch_advance(b, tries, n_active) bind(C, name="mhd_batch_advance")
      import :: c_int, c_ptr
      type(c_ptr), value :: b
      integer(c_int), value :: tries
      integer(c_int), intent(out) :: n_active
    end function

    integer(c_int) function mhd_batch_member_status(b, h, st) bind(C, name="mhd_batch_member_status")
      import :: c_int, c_ptr, mhd_gpu_status
      type(c_ptr), value :: b, h
      type(mhd_gpu_status), intent(out) :: st
    end function
  end interface
end module mhd_gpu_bind
