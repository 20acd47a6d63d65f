!> Fortran binding of the C ABI in canard_gpu.h (iso_c_binding), and drop-in
!> replacements for the reference's per-stage routines.
!>
!> mo_canard_gpu: one interface per entry point of canard_gpu.h, the
!>   constants, and two helpers: c_string (a C string as a Fortran string)
!>   and canard_check (the reference's "write(*,*) msg; stop 1" on an error).
!>
!> mo_canard_gpu_dropin: routines with the reference's argument lists that run
!>   on the device through canard_phase / canard_phase_with:
!>   * t_physics_gpu extends t_physics and overrides calc_viscous_shear_stress
!>     and calc_fluxes (src/mo_physics.f90:216-402), so a driver that declares
!>     type(t_physics_gpu) :: p_physics keeps its call sites;
!>   * gcbc_setup, gcbc_comm, gcbc_update (src/mo_gcbc.f90:133-340) and
!>     spongego (src/mo_sponge.f90:75-88), module procedures of the same names
!>     and arguments, taken instead of mo_gcbc's and mo_sponge's by a `use`.
!>   Each copies the arrays the reference routine reads to the device block
!>   the rank owns, runs the phase and copies back what the routine writes.
!>   canard_step (the whole loop body) needs none of these copies.
module mo_canard_gpu
   use iso_c_binding
   implicit none
   private :: c_strlen

   integer(c_int), parameter :: CANARD_OK = 0, CANARD_ERR_ARG = 1, CANARD_ERR_CUDA = 2, CANARD_ERR_NAN = 3, &
                                CANARD_ERR_TIMEOUT = 4, CANARD_ERR_UNSUPPORTED = 5, CANARD_ERR_STATE = 6, &
                                CANARD_ERR_IO = 7
   integer(c_int32_t), parameter :: CANARD_FP64 = 0, CANARD_FP32_MIXED = 1, CANARD_FP64_FAST = 2
   ! field ids of canard_get_field / canard_set_field
   integer(c_int32_t), parameter :: CANARD_F_QA = 0, CANARD_F_QO = 1, CANARD_F_DE = 2, CANARD_F_P = 3, &
                                    CANARD_F_SS1 = 4, CANARD_F_XIM = 5, CANARD_F_ETM = 6, CANARD_F_ZEM = 7, &
                                    CANARD_F_YACO = 8, CANARD_F_TAU = 9, CANARD_F_DRVA1 = 10, &
                                    CANARD_F_DRVA2 = 11, CANARD_F_DRVA3 = 12, CANARD_F_CM1 = 13, &
                                    CANARD_F_CM2 = 14, CANARD_F_CM3 = 15
   ! phase ids of canard_phase
   integer(c_int32_t), parameter :: CANARD_PH_FILTER = 0, CANARD_PH_COPYQO = 1, CANARD_PH_PRIM = 2, &
                                    CANARD_PH_TIMESTEP = 3, CANARD_PH_VISCOUS = 4, CANARD_PH_FLUXES = 5, &
                                    CANARD_PH_GCBC = 6, CANARD_PH_SPONGE = 7, CANARD_PH_RKUPDATE = 8, &
                                    CANARD_PH_WALL = 9, CANARD_PH_AVERAGE = 10, CANARD_PH_ADVANCE = 11, &
                                    CANARD_PH_MOVEF_A = 12

   !> C canard_block_desc; C nbc[3][2] is Fortran nbc(2,3): side first, direction second
   type, bind(C) :: canard_block_desc
      integer(c_int32_t) :: lxi, let, lze
      integer(c_int32_t) :: nbc(2,3)
      integer(c_int32_t) :: mbcd(2,3)
   end type

   type, bind(C) :: canard_case_desc
      integer(c_int32_t) :: nblocks, viscous
      real(c_double)     :: fltk, fltrbc, reoo, tempoo, amach1, amach2, amach3, timf
      integer(c_int32_t) :: nsmf
      real(c_double)     :: cfl, szco, szth0, szth1, doml0, doml1
   end type

   interface
      ! ---- context life cycle
      integer(c_int) function canard_ctx_create(cases, ncases, blocks, precision, ctx) &
            bind(C, name="canard_ctx_create")
         import
         type(canard_case_desc), intent(in) :: cases(*)
         integer(c_int32_t), value :: ncases
         type(canard_block_desc), intent(in) :: blocks(*)
         integer(c_int32_t), value :: precision
         type(c_ptr), intent(out) :: ctx
      end function
      subroutine canard_ctx_destroy(ctx) bind(C, name="canard_ctx_destroy")
         import
         type(c_ptr), value :: ctx
      end subroutine
      type(c_ptr) function canard_last_error(ctx) bind(C, name="canard_last_error")
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function canard_set_stream(ctx, cuda_stream) bind(C, name="canard_set_stream")
         import
         type(c_ptr), value :: ctx, cuda_stream
      end function
      ! ---- grid, set-up, state
      integer(c_int) function canard_upload_grid(ctx, icase, iblock, xyz) bind(C, name="canard_upload_grid")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, iblock
         real(c_double), intent(in) :: xyz(*)
      end function
      integer(c_int) function canard_set_subdomains(ctx, icase, nblocks, nbpc, mbcd, sub) &
            bind(C, name="canard_set_subdomains")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, nblocks
         integer(c_int32_t), intent(in) :: nbpc(3,*), mbcd(2,3,*), sub(4,*)   ! sub(:,r) = mb, ijkp(1:3)
      end function
      integer(c_int) function canard_setup(ctx) bind(C, name="canard_setup")
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function canard_set_state(ctx, icase, iblock, qa) bind(C, name="canard_set_state")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, iblock
         real(c_double), intent(in) :: qa(*)
      end function
      integer(c_int) function canard_get_state(ctx, icase, iblock, qa) bind(C, name="canard_get_state")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, iblock
         real(c_double), intent(out) :: qa(*)
      end function
      integer(c_int) function canard_get_field(ctx, icase, iblock, field, out, count) &
            bind(C, name="canard_get_field")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, iblock, field
         real(c_double), intent(out) :: out(*)
         integer(c_int64_t), value :: count
      end function
      integer(c_int) function canard_set_field(ctx, icase, iblock, field, in, count) &
            bind(C, name="canard_set_field")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, iblock, field
         real(c_double), intent(in) :: in(*)
         integer(c_int64_t), value :: count
      end function
      ! ---- time loop
      integer(c_int) function canard_step(ctx, nsteps) bind(C, name="canard_step")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: nsteps
      end function
      integer(c_int) function canard_step_host(ctx, nsteps, nblocks, icase, iblock, host) &
            bind(C, name="canard_step_host")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: nsteps, nblocks
         integer(c_int32_t), intent(in) :: icase(*), iblock(*)
         type(c_ptr), intent(in) :: host(*)          ! c_loc of each listed block's qa(0:lmx,5)
      end function
      integer(c_int) function canard_phase(ctx, phase, nk) bind(C, name="canard_phase")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: phase, nk
      end function
      integer(c_int) function canard_phase_with(ctx, phase, nk, dt, umf, dudtmf) bind(C, name="canard_phase_with")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: phase, nk
         real(c_double), value :: dt
         real(c_double), intent(in) :: umf(3), dudtmf(3)
      end function
      integer(c_int) function canard_get_time(ctx, icase, time6) bind(C, name="canard_get_time")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase
         real(c_double), intent(out) :: time6(6)      ! n, ndt, dt, dts, dte, timo
      end function
      integer(c_int) function canard_set_time(ctx, icase, time6) bind(C, name="canard_set_time")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase
         real(c_double), intent(in) :: time6(6)
      end function
      ! ---- restart and grid files (host only)
      integer(c_int) function canard_restart_write_file(path, time6, qa, npts) bind(C, name="canard_restart_write_file")
         import
         character(kind=c_char), intent(in) :: path(*)
         real(c_double), intent(in) :: time6(6), qa(*)
         integer(c_int64_t), value :: npts
      end function
      integer(c_int) function canard_restart_read_file(path, time6, qa, npts) bind(C, name="canard_restart_read_file")
         import
         character(kind=c_char), intent(in) :: path(*)
         real(c_double), intent(out) :: time6(6), qa(*)
         integer(c_int64_t), value :: npts
      end function
      integer(c_int) function canard_grid_write_file(path, xyz, npts) bind(C, name="canard_grid_write_file")
         import
         character(kind=c_char), intent(in) :: path(*)
         real(c_double), intent(in) :: xyz(*)
         integer(c_int64_t), value :: npts
      end function
      integer(c_int) function canard_grid_read_file(path, xyz, npts) bind(C, name="canard_grid_read_file")
         import
         character(kind=c_char), intent(in) :: path(*)
         real(c_double), intent(out) :: xyz(*)
         integer(c_int64_t), value :: npts
      end function
      integer(c_int) function canard_write_restart(ctx, icase, iblock, path) bind(C, name="canard_write_restart")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, iblock
         character(kind=c_char), intent(in) :: path(*)
      end function
      integer(c_int) function canard_read_restart(ctx, icase, iblock, path) bind(C, name="canard_read_restart")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase, iblock
         character(kind=c_char), intent(in) :: path(*)
      end function
      integer(c_int) function canard_restart_compare(path1, path2, npts, wtol, report_path, nreported) &
            bind(C, name="canard_restart_compare")
         import
         character(kind=c_char), intent(in) :: path1(*), path2(*), report_path(*)
         integer(c_int64_t), value :: npts
         real(c_double), value :: wtol
         integer(c_int64_t), intent(out) :: nreported
      end function
      ! ---- host-side plans of the junction averaging and the exchanges
      integer(c_int) function canard_average_host(nranks, ranks, nblocks, nbpc, mbcd, sub, qa) &
            bind(C, name="canard_average_host")
         import
         integer(c_int32_t), value :: nranks
         type(canard_block_desc), intent(in) :: ranks(*)
         integer(c_int32_t), value :: nblocks
         integer(c_int32_t), intent(in) :: nbpc(*), mbcd(*), sub(*)
         type(c_ptr), intent(in) :: qa(*)             ! c_loc of each rank's qa(0:lmx,5)
      end function
      integer(c_int) function canard_plan_export(nranks, ranks, nblocks, nbpc, mbcd, sub, kind, out, cap, n) &
            bind(C, name="canard_plan_export")
         import
         integer(c_int32_t), value :: nranks
         type(canard_block_desc), intent(in) :: ranks(*)
         integer(c_int32_t), value :: nblocks
         integer(c_int32_t), intent(in) :: nbpc(*), mbcd(*), sub(*)
         integer(c_int32_t), value :: kind
         integer(c_int64_t), intent(out) :: out(*)
         integer(c_int64_t), value :: cap
         integer(c_int64_t), intent(out) :: n
      end function
      ! ---- recording and Tecplot output
      integer(c_int) function canard_record_enable(ctx, on) bind(C, name="canard_record_enable")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: on
      end function
      integer(c_int) function canard_record_accumulate(ctx) bind(C, name="canard_record_accumulate")
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function canard_record_output(ctx, icase, vart, time_out) bind(C, name="canard_record_output")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: icase
         type(c_ptr), intent(in) :: vart(*)           ! c_loc of each block's real(c_float) array
         real(c_double), intent(out) :: time_out
      end function
      integer(c_int) function canard_plt_write(path, n, nblocks, dims, time, data) bind(C, name="canard_plt_write")
         import
         character(kind=c_char), intent(in) :: path(*)
         integer(c_int32_t), value :: n, nblocks
         integer(c_int32_t), intent(in) :: dims(*)
         real(c_double), value :: time
         type(c_ptr), intent(in) :: data(*)
      end function
      ! ---- t_numerics unit operations on host arrays
      integer(c_int) function canard_mpigo(ctx, fields, ncols, nt, nrt, n45, itag, m) bind(C, name="canard_mpigo")
         import
         type(c_ptr), value :: ctx
         type(c_ptr), intent(in) :: fields(*)         ! c_loc of each block's rfield(0:lmx,ncols)
         integer(c_int32_t), value :: ncols, nt, nrt, n45, itag, m
      end function
      integer(c_int) function canard_deriv(ctx, iblock, fin, fout, nn, m) bind(C, name="canard_deriv")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: iblock
         real(c_double), intent(in) :: fin(*)
         real(c_double), intent(out) :: fout(*)
         integer(c_int32_t), value :: nn, m
      end function
      integer(c_int) function canard_filte(ctx, iblock, f, inn, m) bind(C, name="canard_filte")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: iblock
         real(c_double), intent(inout) :: f(*)
         integer(c_int32_t), value :: inn, m
      end function
      ! ---- coefficient tables (host only)
      integer(c_int) function canard_coeffs(fltk, fltrbc, out150) bind(C, name="canard_coeffs")
         import
         real(c_double), value :: fltk, fltrbc
         real(c_double), intent(out) :: out150(150)
      end function
      integer(c_int) function canard_penta(fltk, fltrbc, n, ns, ne, nt, xu, xl) bind(C, name="canard_penta")
         import
         real(c_double), value :: fltk, fltrbc
         integer(c_int32_t), value :: n, ns, ne, nt
         real(c_double), intent(out) :: xu(*), xl(*)
      end function
      integer(c_int) function canard_version() bind(C, name="canard_version")
         import
      end function
      ! ---- tuning, measurement, observability
      integer(c_int) function canard_line_bench(ctx, op, nn, nfields, fin, fout, reps, ms_per_launch) &
            bind(C, name="canard_line_bench")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: op, nn, nfields
         real(c_double), intent(in) :: fin(*)
         real(c_double), intent(out) :: fout(*)
         integer(c_int32_t), value :: reps
         real(c_double), intent(out) :: ms_per_launch
      end function
      integer(c_int) function canard_autotune(ctx, reps, report, nmax) bind(C, name="canard_autotune")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: reps
         real(c_double), intent(out) :: report(*)
         integer(c_int32_t), value :: nmax
      end function
      integer(c_int) function canard_set_line_kind(ctx, group, dir, kind, chunks) bind(C, name="canard_set_line_kind")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: group, dir, kind, chunks
      end function
      integer(c_int) function canard_set_timers(ctx, on) bind(C, name="canard_set_timers")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: on
      end function
      integer(c_int) function canard_get_timers(ctx, ms, launches, bytes, nmax) bind(C, name="canard_get_timers")
         import
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: ms(*), launches(*), bytes(*)
         integer(c_int32_t), value :: nmax
      end function
      type(c_ptr) function canard_timer_name(family) bind(C, name="canard_timer_name")
         import
         integer(c_int32_t), value :: family
      end function
      integer(c_int) function canard_launch_count(ctx, count) bind(C, name="canard_launch_count")
         import
         type(c_ptr), value :: ctx
         integer(c_int64_t), intent(out) :: count
      end function
      integer(c_int) function canard_selftest_wait(ctx, seconds) bind(C, name="canard_selftest_wait")
         import
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: seconds
      end function
      integer(c_int) function canard_set_graphs(ctx, on) bind(C, name="canard_set_graphs")
         import
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: on
      end function
      ! ---- the derivative without device allocation (device arrays, e.g. from OpenACC)
      integer(c_int) function canard_deriv_noalloc(d_in, d_out, lxi, let, lze, pitch, nn, nbc0, nbc1, fltk, &
                                                   fltrbc, stream) bind(C, name="canard_deriv_noalloc")
         import
         type(c_ptr), value :: d_in, d_out
         integer(c_int32_t), value :: lxi, let, lze, pitch, nn, nbc0, nbc1
         real(c_double), value :: fltk, fltrbc
         type(c_ptr), value :: stream
      end function
      integer(c_int) function canard_deriv_noalloc_status(stream) bind(C, name="canard_deriv_noalloc_status")
         import
         type(c_ptr), value :: stream
      end function
      ! ---- libc, for c_string
      integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
         import
         type(c_ptr), value :: s
      end function
   end interface

contains

   !> The C string at p (canard_last_error, canard_timer_name) as a Fortran string.
   function c_string(p) result(s)
      type(c_ptr), intent(in) :: p
      character(len=:), allocatable :: s
      character(kind=c_char), pointer :: a(:)
      integer :: n, i
      if (.not. c_associated(p)) then
         s = ''
         return
      end if
      n = int(c_strlen(p))
      call c_f_pointer(p, a, [n])
      allocate(character(len=n) :: s)
      do i = 1, n
         s(i:i) = a(i)
      end do
   end function c_string

   !> Stops with the library's message on an error code, as the reference stops
   !> on its own errors (write(*,*) msg; stop 1).
   subroutine canard_check(rc, ctx, where)
      integer(c_int), intent(in) :: rc
      type(c_ptr), intent(in) :: ctx
      character(len=*), intent(in) :: where
      if (rc == CANARD_OK) return
      if (rc == CANARD_ERR_NAN) then
         write(*,*) 'Canard: Overflow.'
      else
         write(*,*) 'Canard GPU (', where, '): ', c_string(canard_last_error(ctx))
      end if
      stop 1
   end subroutine canard_check

end module mo_canard_gpu


module mo_canard_gpu_dropin
   use iso_c_binding
   use mo_kind,      only : ni, nr
   use mo_domdcomp,  only : t_domdcomp
   use mo_numerics,  only : t_numerics
   use mo_grid,      only : t_grid
   use mo_physics,   only : t_physics
   use mo_canard_gpu
   implicit none
   private
   public :: t_physics_gpu, canard_gpu_attach, gcbc_setup, gcbc_comm, gcbc_update, spongego

   !> the context and the block of it that holds this rank's sub-domain
   type(c_ptr), save        :: gpu_ctx = c_null_ptr
   integer(c_int32_t), save :: gpu_case = 0, gpu_block = 0

   !> t_physics with the viscous stresses and the fluxes on the device
   type, extends(t_physics) :: t_physics_gpu
   contains
      procedure, public :: calc_viscous_shear_stress => calc_viscous_shear_stress_gpu
      procedure, public :: calc_fluxes => calc_fluxes_gpu
   end type t_physics_gpu

contains

   !> Names the context (created, grid uploaded, canard_setup done) and the
   !> block (0-based) that holds this rank's sub-domain.
   subroutine canard_gpu_attach(ctx, icase, iblock)
      type(c_ptr), intent(in) :: ctx
      integer(c_int32_t), intent(in) :: icase, iblock
      gpu_ctx = ctx
      gpu_case = icase
      gpu_block = iblock
   end subroutine canard_gpu_attach

   subroutine put(field, a, n)
      integer(c_int32_t), intent(in) :: field
      real(kind=nr), intent(in) :: a(*)
      integer(c_int64_t), intent(in) :: n
      call canard_check(canard_set_field(gpu_ctx, gpu_case, gpu_block, field, a, n), gpu_ctx, 'set_field')
   end subroutine put

   subroutine get(field, a, n)
      integer(c_int32_t), intent(in) :: field
      real(kind=nr), intent(inout) :: a(*)
      integer(c_int64_t), intent(in) :: n
      call canard_check(canard_get_field(gpu_ctx, gpu_case, gpu_block, field, a, n), gpu_ctx, 'get_field')
   end subroutine get

   !> src/mo_physics.f90:216-301: de(:,2:5) = u, v, w, gamma p / rho and ssk
   !> in; de(:,1) = ssk out, the stresses and heat fluxes stay on the device
   !> for calc_fluxes.
   subroutine calc_viscous_shear_stress_gpu(this, p_domdcomp, p_numerics, p_grid, de, ssk)
      class(t_physics_gpu), intent(inout) :: this
      type(t_domdcomp), intent(in)    :: p_domdcomp
      type(t_numerics), intent(inout) :: p_numerics
      type(t_grid),     intent(in)    :: p_grid
      real(kind=nr), dimension(0:p_domdcomp%lmx,5), intent(inout) :: de
      real(kind=nr), dimension(0:p_domdcomp%lmx),   intent(in)    :: ssk
      integer(c_int64_t) :: n
      n = int(p_domdcomp%lmx, c_int64_t) + 1
      call put(CANARD_F_DE, de, 5 * n)
      call put(CANARD_F_SS1, ssk, n)
      call canard_check(canard_phase(gpu_ctx, CANARD_PH_VISCOUS, 1_c_int32_t), gpu_ctx, 'calc_viscous_shear_stress')
      call get(CANARD_F_DE, de, 5 * n)
   end subroutine calc_viscous_shear_stress_gpu

   !> src/mo_physics.f90:306-402 with the frame velocity this%umf of the stage
   !> (set by movef): de out = the divergence of the fluxes.
   subroutine calc_fluxes_gpu(this, p_domdcomp, p_numerics, p_grid, qa, p, de)
      class(t_physics_gpu), intent(inout) :: this
      type(t_domdcomp), intent(in)    :: p_domdcomp
      type(t_numerics), intent(inout) :: p_numerics
      type(t_grid),     intent(in)    :: p_grid
      real(kind=nr), dimension(0:p_domdcomp%lmx,5), intent(in)    :: qa
      real(kind=nr), dimension(0:p_domdcomp%lmx),   intent(in)    :: p
      real(kind=nr), dimension(0:p_domdcomp%lmx,5), intent(inout) :: de
      integer(c_int64_t) :: n
      real(c_double) :: umf(3), dudtmf(3)
      n = int(p_domdcomp%lmx, c_int64_t) + 1
      umf = this%umf
      dudtmf = this%dudtmf
      call put(CANARD_F_QA, qa, 5 * n)
      call put(CANARD_F_P, p, n)
      call put(CANARD_F_DE, de, 5 * n)
      call canard_check(canard_phase_with(gpu_ctx, CANARD_PH_FLUXES, 1_c_int32_t, 0.0_c_double, umf, dudtmf), &
                        gpu_ctx, 'calc_fluxes')
      call get(CANARD_F_DE, de, 5 * n)
   end subroutine calc_fluxes_gpu

   !> src/mo_gcbc.f90:133-184. The device forms the characteristic values
   !> inside gcbc_update, from the qa, p and de it receives there; the driver
   !> calls the three routines back to back with the same arrays.
   subroutine gcbc_setup(p_domdcomp, p_numerics, p_grid, qa, p, de, umf)
      type(t_domdcomp), intent(in)    :: p_domdcomp
      type(t_numerics), intent(inout) :: p_numerics
      type(t_grid),     intent(in)    :: p_grid
      real(kind=nr), dimension(0:p_domdcomp%lmx,5), intent(in) :: qa
      real(kind=nr), dimension(0:p_domdcomp%lmx),   intent(in) :: p
      real(kind=nr), dimension(0:p_domdcomp%lmx,5), intent(in) :: de
      real(kind=nr), dimension(3), intent(in) :: umf
   end subroutine gcbc_setup

   !> src/mo_gcbc.f90:186-220: on one device the drva exchange across curved
   !> interfaces is part of the device's GCBC phase.
   subroutine gcbc_comm(p_domdcomp, p_numerics)
      type(t_domdcomp), intent(in)    :: p_domdcomp
      type(t_numerics), intent(inout) :: p_numerics
   end subroutine gcbc_comm

   !> src/mo_gcbc.f90:222-340 (with the set-up and the exchange): de is
   !> updated on the non-reflecting, wall and curved-interface faces.
   subroutine gcbc_update(p_domdcomp, p_numerics, p_grid, qa, p, de, nkrk, dt, umf, dudtmf)
      type(t_domdcomp), intent(in)    :: p_domdcomp
      type(t_numerics), intent(inout) :: p_numerics
      type(t_grid),     intent(in)    :: p_grid
      real(kind=nr), dimension(0:p_domdcomp%lmx,5), intent(in)    :: qa
      real(kind=nr), dimension(0:p_domdcomp%lmx),   intent(in)    :: p
      real(kind=nr), dimension(0:p_domdcomp%lmx,5), intent(inout) :: de
      integer(kind=ni), intent(in) :: nkrk
      real(kind=nr), intent(in) :: dt
      real(kind=nr), dimension(3), intent(in) :: umf, dudtmf
      integer(c_int64_t) :: n
      real(c_double) :: u(3), a(3)
      n = int(p_domdcomp%lmx, c_int64_t) + 1
      u = umf
      a = dudtmf
      call put(CANARD_F_QA, qa, 5 * n)
      call put(CANARD_F_P, p, n)
      call put(CANARD_F_DE, de, 5 * n)
      call canard_check(canard_phase_with(gpu_ctx, CANARD_PH_GCBC, 1_c_int32_t, real(dt, c_double), u, a), &
                        gpu_ctx, 'gcbc_update')
      call get(CANARD_F_DE, de, 5 * n)
   end subroutine gcbc_update

   !> src/mo_sponge.f90:75-88: de += sigma / yaco (q - q_inf) on the sponge points.
   subroutine spongego(lmx, qa, de)
      integer(kind=ni), intent(in) :: lmx
      real(kind=nr), dimension(0:lmx,5), intent(in)    :: qa
      real(kind=nr), dimension(0:lmx,5), intent(inout) :: de
      integer(c_int64_t) :: n
      n = int(lmx, c_int64_t) + 1
      call put(CANARD_F_QA, qa, 5 * n)
      call put(CANARD_F_DE, de, 5 * n)
      call canard_check(canard_phase(gpu_ctx, CANARD_PH_SPONGE, 1_c_int32_t), gpu_ctx, 'spongego')
      call get(CANARD_F_DE, de, 5 * n)
   end subroutine spongego

end module mo_canard_gpu_dropin
