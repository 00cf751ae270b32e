!===============================================================================
! mod_solver_gpu.f90 - iso_c_binding interface to libeafcg.so (the B200
! pressure-correction CG) and a drop-in replacement for cg_3d_mpi.
!
! The reference call in solve_pressure_correction
! (src/mod_pressure_3d.f90:316-318)
!     call cg_3d_mpi(aW, aE, aS, aN, aB, aT, aP, Su, sh%pp, m, &
!                    cfg%max_inner_pres, SOR_TOL_PRESSURE, cg_res, n_iter_cg)
! becomes
!     call cg_3d_gpu(aW, aE, aS, aN, aB, aT, aP, Su, sh%pp, m, &
!                    cfg%max_inner_pres, SOR_TOL_PRESSURE, cg_res, n_iter_cg)
! with the same dummies and meaning as cg_3d_mpi (src/mod_solver_3d.f90:
! 485-496). The workspace arrays are contiguous allocatables
! (src/mod_workspace.f90:120-126), so they pass to the C entry point without
! copies. Not compiled in this repository's build (no Fortran compiler is
! available where it is built); link with -L<dir> -leafcg.
!
! The same module replaces the line-by-line TDMA and the transport residual
! of mod_solver_3d (tdma_3d_mpi, :252-366; compute_residual_3d_mpi,
! :625-694) for their callers in momentum, energy, species, turbulence,
! radiation and continuity (e.g. src/mod_momentum_3d.f90:326-329):
!     residual = compute_residual_3d_gpu(aW, ..., Su, vel, m)
!     call tdma_3d_gpu(aW, ..., Su, vel, m, cfg%max_inner_mom)
! and the post-CG corrections of solve_pressure_correction
! (src/mod_pressure_3d.f90:333-397 with correct_velocities :689-746) become
! one call of pressure_correct_gpu (fill an eaf_pcorr_fields with c_loc of
! the arrays; see its comment), and the assembly of the pressure-correction
! equation before the CG (src/mod_pressure_3d.f90:135-310 with
! apply_pressure_bc, src/mod_boundary_3d.f90:180-277) one call of
! pressure_assemble_gpu (an eaf_assembly_fields).
!===============================================================================
module mod_solver_gpu
    use iso_c_binding
    implicit none
    private
    public :: cg_3d_gpu, cg_3d_gpu_mixed, cg_gpu_release
    public :: tdma_3d_gpu, compute_residual_3d_gpu
    public :: eaf_cg_create, eaf_cg_destroy, eaf_cg_solve_f64, eaf_cg_solve_mixed
    public :: eaf_tdma_3d_f64, eaf_residual_3d_f64
    public :: eaf_phase_fields, eaf_pcorr_fields, pressure_correct_gpu
    public :: eaf_phase_state, eaf_assembly_fields, pressure_assemble_gpu
    public :: pressure_step_gpu
    public :: cg_3d_gpu_mpi

    integer(c_int), parameter, public :: EAF_OK = 0, EAF_ENONFINITE = 3

    ! Mirrors of eaf_phase_fields_t / eaf_pcorr_fields_t (include/eafcg.h):
    ! c_loc of the phase and workspace arrays, c_null_ptr for the gas when
    ! it is not in the pressure equation.
    type, bind(C) :: eaf_phase_fields
        type(c_ptr) :: alpha, aP_ur, aP_uth, aP_uz, ur, uth, uz
    end type eaf_phase_fields

    type, bind(C) :: eaf_pcorr_fields
        type(c_ptr) :: pp, Fs_r, Fs_th, Fs_z, ac_r, ac_th, ac_z
        type(c_ptr) :: Fc_r, Fc_th, Fc_z, vol, r, theta, z, p
        type(eaf_phase_fields) :: liq, gas
        type(c_ptr) :: lk_r, lk_th, lk_z, cell_type, act_l, act_g
        integer(c_int) :: has_gas
        real(c_double) :: alpha_p
    end type eaf_pcorr_fields

    ! Mirrors of eaf_phase_state_t / eaf_assembly_fields_t: the inputs of
    ! the assembly (c_loc of the mesh, state and mask arrays; outlet is the
    ! out_mask of apply_pressure_bc, nonzero where an electrode hole covers a
    ! top-layer cell; act_l / act_g and liq_room as the caller computes them
    ! for the phase loops), the switches and scalars, and the outputs.
    type, bind(C) :: eaf_phase_state
        type(c_ptr) :: alpha, rho, ur, uth, uz, aP_ur, aP_uth, aP_uz
    end type eaf_phase_state

    type, bind(C) :: eaf_assembly_fields
        type(c_ptr) :: cell_type, outlet, act_l, act_g
        type(c_ptr) :: vol, Ar, Ath, Az, r, theta, z, p, liq_room
        type(eaf_phase_state) :: liq, gas
        type(c_ptr) :: liq_T, gas_T_old
        integer(c_int) :: liq_room_valid, gas_in_poisson, gas_compressibility
        real(c_double) :: dt, rho_gas, T_ambient, beta_expansion
        type(c_ptr) :: aW, aE, aS, aN, aB, aT, aP, Su, pp
        type(c_ptr) :: Fs_r, Fs_th, Fs_z, ac_r, ac_th, ac_z, Fc_r, Fc_th, Fc_z
        type(c_ptr) :: lk_r, lk_th, lk_z
    end type eaf_assembly_fields

    interface
        integer(c_int) function eaf_cg_create(h, nr, nth, nz, device) &
                bind(C, name="eaf_cg_create")
            import :: c_int, c_ptr
            type(c_ptr), intent(out) :: h
            integer(c_int), value :: nr, nth, nz, device
        end function eaf_cg_create

        integer(c_int) function eaf_cg_destroy(h) bind(C, name="eaf_cg_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function eaf_cg_destroy

        integer(c_int) function eaf_cg_solve_f64(h, aW, aE, aS, aN, aB, aT, aP, &
                Su, phi, max_iter, tol, residual, n_iter) &
                bind(C, name="eaf_cg_solve_f64")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: aW(*), aE(*), aS(*), aN(*)
            real(c_double), intent(in) :: aB(*), aT(*), aP(*), Su(*)
            real(c_double), intent(inout) :: phi(*)
            integer(c_int), value :: max_iter
            real(c_double), value :: tol
            real(c_double), intent(out) :: residual
            integer(c_int), intent(out) :: n_iter
        end function eaf_cg_solve_f64

        integer(c_int) function eaf_cg_solve_mixed(h, aW, aE, aS, aN, aB, aT, &
                aP, Su, phi, max_outer, max_inner, tol, inner_tol, residual, &
                n_iter, n_outer) bind(C, name="eaf_cg_solve_mixed")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: aW(*), aE(*), aS(*), aN(*)
            real(c_double), intent(in) :: aB(*), aT(*), aP(*), Su(*)
            real(c_double), intent(inout) :: phi(*)
            integer(c_int), value :: max_outer, max_inner
            real(c_double), value :: tol, inner_tol
            real(c_double), intent(out) :: residual
            integer(c_int), intent(out) :: n_iter, n_outer
        end function eaf_cg_solve_mixed

        integer(c_int) function eaf_tdma_3d_f64(h, aW, aE, aS, aN, aB, aT, aP, &
                Su, phi, n_sweep) bind(C, name="eaf_tdma_3d_f64")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: aW(*), aE(*), aS(*), aN(*)
            real(c_double), intent(in) :: aB(*), aT(*), aP(*), Su(*)
            real(c_double), intent(inout) :: phi(*)
            integer(c_int), value :: n_sweep
        end function eaf_tdma_3d_f64

        integer(c_int) function eaf_residual_3d_f64(h, aW, aE, aS, aN, aB, aT, aP, &
                Su, phi, residual) bind(C, name="eaf_residual_3d_f64")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: aW(*), aE(*), aS(*), aN(*)
            real(c_double), intent(in) :: aB(*), aT(*), aP(*), Su(*)
            real(c_double), intent(in) :: phi(*)
            real(c_double), intent(out) :: residual
        end function eaf_residual_3d_f64

        integer(c_int) function eaf_mr_block(nr, nth, nz, grid, coords, loc, start) &
                bind(C, name="eaf_mr_block")
            import :: c_int
            integer(c_int), value :: nr, nth, nz
            integer(c_int), intent(in) :: grid(3), coords(3)
            integer(c_int), intent(out) :: loc(3), start(3)
        end function eaf_mr_block

        integer(c_long_long) function eaf_mr_pack_count(grid, coords, loc) &
                bind(C, name="eaf_mr_pack_count")
            import :: c_int, c_long_long
            integer(c_int), intent(in) :: grid(3), coords(3), loc(3)
        end function eaf_mr_pack_count

        integer(c_long_long) function eaf_mr_unpack_count(nr, nz, start, loc) &
                bind(C, name="eaf_mr_unpack_count")
            import :: c_int, c_long_long
            integer(c_int), value :: nr, nz
            integer(c_int), intent(in) :: start(3), loc(3)
        end function eaf_mr_unpack_count

        integer(c_int) function eaf_mr_pack(local, grid, coords, loc, buf) &
                bind(C, name="eaf_mr_pack")
            import :: c_int, c_double
            real(c_double), intent(in) :: local(*)
            integer(c_int), intent(in) :: grid(3), coords(3), loc(3)
            real(c_double), intent(out) :: buf(*)
        end function eaf_mr_pack

        integer(c_int) function eaf_mr_place(global, nr, nth, nz, grid, coords, loc, &
                start, buf) bind(C, name="eaf_mr_place")
            import :: c_int, c_double
            real(c_double), intent(inout) :: global(*)
            integer(c_int), value :: nr, nth, nz
            integer(c_int), intent(in) :: grid(3), coords(3), loc(3), start(3)
            real(c_double), intent(in) :: buf(*)
        end function eaf_mr_place

        integer(c_int) function eaf_mr_extract(global, nr, nth, nz, loc, start, buf) &
                bind(C, name="eaf_mr_extract")
            import :: c_int, c_double
            real(c_double), intent(in) :: global(*)
            integer(c_int), value :: nr, nth, nz
            integer(c_int), intent(in) :: loc(3), start(3)
            real(c_double), intent(out) :: buf(*)
        end function eaf_mr_extract

        integer(c_int) function eaf_mr_unpack(local, nr, nz, loc, start, buf) &
                bind(C, name="eaf_mr_unpack")
            import :: c_int, c_double
            real(c_double), intent(inout) :: local(*)
            integer(c_int), value :: nr, nz
            integer(c_int), intent(in) :: loc(3), start(3)
            real(c_double), intent(in) :: buf(*)
        end function eaf_mr_unpack

        integer(c_int) function eaf_pressure_correct_f64(h, f) &
                bind(C, name="eaf_pressure_correct_f64")
            import :: c_int, c_ptr, eaf_pcorr_fields
            type(c_ptr), value :: h
            type(eaf_pcorr_fields), intent(in) :: f
        end function eaf_pressure_correct_f64

        integer(c_int) function eaf_pressure_assemble_f64(h, f, residual) &
                bind(C, name="eaf_pressure_assemble_f64")
            import :: c_int, c_ptr, c_double, eaf_assembly_fields
            type(c_ptr), value :: h
            type(eaf_assembly_fields), intent(in) :: f
            real(c_double), intent(out) :: residual
        end function eaf_pressure_assemble_f64

        integer(c_int) function eaf_pressure_step_f64(h, f, alpha_p, max_iter, tol, &
                residual, cg_res, n_iter) bind(C, name="eaf_pressure_step_f64")
            import :: c_int, c_ptr, c_double, eaf_assembly_fields
            type(c_ptr), value :: h
            type(eaf_assembly_fields), intent(in) :: f
            real(c_double), value :: alpha_p, tol
            integer(c_int), value :: max_iter
            real(c_double), intent(out) :: residual, cg_res
            integer(c_int), intent(out) :: n_iter
        end function eaf_pressure_step_f64
    end interface

    ! One handle per mesh size, kept across SIMPLE iterations like the
    ! reference's persistent workspace (src/mod_workspace.f90:120-144).
    type(c_ptr), save :: handle = c_null_ptr
    integer, save :: h_nr = -1, h_nth = -1, h_nz = -1

contains

    subroutine ensure_handle(nr, nth, nz)
        integer, intent(in) :: nr, nth, nz
        integer(c_int) :: st
        if (c_associated(handle) .and. nr == h_nr .and. nth == h_nth &
            .and. nz == h_nz) return
        if (c_associated(handle)) st = eaf_cg_destroy(handle)
        st = eaf_cg_create(handle, int(nr, c_int), int(nth, c_int), &
                           int(nz, c_int), 0_c_int)
        if (st /= EAF_OK) error stop 'eaf_cg_create failed'
        h_nr = nr; h_nth = nth; h_nz = nz
    end subroutine ensure_handle

    ! Same dummies as cg_3d_mpi; serial meshes only (the whole theta x z
    ! domain on one GPU). A NaN residual is returned like the reference's.
    subroutine cg_3d_gpu(aW, aE, aS, aN, aB, aT, aP, Su, phi, m, &
                         max_iter, tol, residual, n_iter)
        use mod_constants, only: dp
        use mod_types_3d, only: mesh_t
        real(dp), intent(in), contiguous  :: aW(-1:,-1:,-1:), aE(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aS(-1:,-1:,-1:), aN(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aB(-1:,-1:,-1:), aT(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aP(-1:,-1:,-1:), Su(-1:,-1:,-1:)
        real(dp), intent(inout), contiguous :: phi(-1:,-1:,-1:)
        type(mesh_t), intent(in) :: m
        integer, intent(in)      :: max_iter
        real(dp), intent(in)     :: tol
        real(dp), intent(out)    :: residual
        integer, intent(out)     :: n_iter
        integer(c_int) :: st, nit
        real(c_double) :: res
        if (m%is_parallel) error stop 'cg_3d_gpu: decomposed meshes are not supported'
        call ensure_handle(m%nr, m%ntheta, m%nz)
        st = eaf_cg_solve_f64(handle, aW, aE, aS, aN, aB, aT, aP, Su, phi, &
                              int(max_iter, c_int), real(tol, c_double), res, nit)
        if (st /= EAF_OK .and. st /= EAF_ENONFINITE) error stop 'eaf_cg_solve_f64 failed'
        residual = res
        n_iter = nit
    end subroutine cg_3d_gpu

    ! Mixed FP32/FP64 form (no reference counterpart): same arrays.
    subroutine cg_3d_gpu_mixed(aW, aE, aS, aN, aB, aT, aP, Su, phi, m, &
                               tol, residual, n_iter)
        use mod_constants, only: dp
        use mod_types_3d, only: mesh_t
        real(dp), intent(in), contiguous  :: aW(-1:,-1:,-1:), aE(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aS(-1:,-1:,-1:), aN(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aB(-1:,-1:,-1:), aT(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aP(-1:,-1:,-1:), Su(-1:,-1:,-1:)
        real(dp), intent(inout), contiguous :: phi(-1:,-1:,-1:)
        type(mesh_t), intent(in) :: m
        real(dp), intent(in)     :: tol
        real(dp), intent(out)    :: residual
        integer, intent(out)     :: n_iter
        integer(c_int) :: st, nit, nout
        real(c_double) :: res
        if (m%is_parallel) error stop 'cg_3d_gpu_mixed: decomposed meshes are not supported'
        call ensure_handle(m%nr, m%ntheta, m%nz)
        st = eaf_cg_solve_mixed(handle, aW, aE, aS, aN, aB, aT, aP, Su, phi, &
                                200_c_int, 100000_c_int, real(tol, c_double), &
                                0.1_c_double, res, nit, nout)
        if (st /= EAF_OK .and. st /= EAF_ENONFINITE) error stop 'eaf_cg_solve_mixed failed'
        residual = res
        n_iter = nit
    end subroutine cg_3d_gpu_mixed

    ! Same dummies as tdma_3d_mpi; serial meshes only. phi comes back
    ! bit-identical to the serial routine's.
    subroutine tdma_3d_gpu(aW, aE, aS, aN, aB, aT, aP, Su, phi, m, n_sweep)
        use mod_constants, only: dp
        use mod_types_3d, only: mesh_t
        real(dp), intent(in), contiguous  :: aW(-1:,-1:,-1:), aE(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aS(-1:,-1:,-1:), aN(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aB(-1:,-1:,-1:), aT(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aP(-1:,-1:,-1:), Su(-1:,-1:,-1:)
        real(dp), intent(inout), contiguous :: phi(-1:,-1:,-1:)
        type(mesh_t), intent(in) :: m
        integer, intent(in)      :: n_sweep
        integer(c_int) :: st
        if (m%is_parallel) error stop 'tdma_3d_gpu: decomposed meshes are not supported'
        call ensure_handle(m%nr, m%ntheta, m%nz)
        st = eaf_tdma_3d_f64(handle, aW, aE, aS, aN, aB, aT, aP, Su, phi, &
                             int(n_sweep, c_int))
        if (st /= EAF_OK) error stop 'eaf_tdma_3d_f64 failed'
    end subroutine tdma_3d_gpu

    ! Same dummies and result as compute_residual_3d_mpi; serial meshes only.
    function compute_residual_3d_gpu(aW, aE, aS, aN, aB, aT, aP, Su, phi, m) result(res)
        use mod_constants, only: dp
        use mod_types_3d, only: mesh_t
        real(dp), intent(in), contiguous :: aW(-1:,-1:,-1:), aE(-1:,-1:,-1:)
        real(dp), intent(in), contiguous :: aS(-1:,-1:,-1:), aN(-1:,-1:,-1:)
        real(dp), intent(in), contiguous :: aB(-1:,-1:,-1:), aT(-1:,-1:,-1:)
        real(dp), intent(in), contiguous :: aP(-1:,-1:,-1:), Su(-1:,-1:,-1:)
        real(dp), intent(in), contiguous :: phi(-1:,-1:,-1:)
        type(mesh_t), intent(in) :: m
        real(dp) :: res
        integer(c_int) :: st
        real(c_double) :: r
        if (m%is_parallel) error stop 'compute_residual_3d_gpu: decomposed meshes are not supported'
        call ensure_handle(m%nr, m%ntheta, m%nz)
        st = eaf_residual_3d_f64(handle, aW, aE, aS, aN, aB, aT, aP, Su, phi, r)
        if (st /= EAF_OK) error stop 'eaf_residual_3d_f64 failed'
        res = r
    end function compute_residual_3d_gpu

    ! Replaces src/mod_pressure_3d.f90:333-397 (flux export, halo refresh of
    ! the fluxes and link flags, correct_velocities of both phases, pressure
    ! update and clamp, sealed cells, halo refresh of p): the caller fills
    ! f with c_loc of sh%pp, Fs_*, ac_*, ws_Fc_*, m%vol, m%r, m%theta, m%z,
    ! sh%p, the phase arrays (liq, gas), ws_Fc_lk_*, m%cell_type, act_l and
    ! act_g (default logicals), has_gas and cfg%alpha_p. Bit-identical to the
    ! serial Fortran. Serial meshes only.
    subroutine pressure_correct_gpu(f, m)
        use mod_types_3d, only: mesh_t
        type(eaf_pcorr_fields), intent(in) :: f
        type(mesh_t), intent(in) :: m
        integer(c_int) :: st
        if (m%is_parallel) error stop 'pressure_correct_gpu: decomposed meshes are not supported'
        call ensure_handle(m%nr, m%ntheta, m%nz)
        st = eaf_pressure_correct_f64(handle, f)
        if (st /= EAF_OK) error stop 'eaf_pressure_correct_f64 failed'
    end subroutine pressure_correct_gpu

    ! Replaces src/mod_pressure_3d.f90:135-310 up to the CG (coefficient
    ! arrays and pp zeroed, cell gradients of both phases, the liquid's and
    ! the gas's face contributions with the exported Fs_*, ac_* and link
    ! flags, the gas compressibility source, trivial rows and the diagonal,
    ! apply_pressure_bc, the continuity residual sum|Su| / flux_ref): the
    ! caller fills f with c_loc of the workspace and state arrays, the
    ! switches (ws_liq_room_valid, cfg%gas_in_poisson .and.
    ! cfg%solve_multiphase, cfg%gas_compressibility .and.
    ! cfg%solve_multiphase) and scalars (dt, RHO_GAS, T_AMBIENT,
    ! BETA_EXPANSION). Every array is bit-identical to the serial Fortran;
    ! the residual agrees to 1e-12 relative (its sums are associated per
    ! block). Serial meshes only.
    subroutine pressure_assemble_gpu(f, m, residual)
        use mod_types_3d, only: mesh_t
        type(eaf_assembly_fields), intent(in) :: f
        type(mesh_t), intent(in) :: m
        real(c_double), intent(out) :: residual
        integer(c_int) :: st
        if (m%is_parallel) error stop 'pressure_assemble_gpu: decomposed meshes are not supported'
        call ensure_handle(m%nr, m%ntheta, m%nz)
        st = eaf_pressure_assemble_f64(handle, f, residual)
        if (st /= EAF_OK) error stop 'eaf_pressure_assemble_f64 failed'
    end subroutine pressure_assemble_gpu

    ! The serial numerics of solve_pressure_correction (src/mod_pressure_3d.f90:
    ! 135-397) in one call: pressure_assemble_gpu, the CG into sh%pp
    ! (cfg%max_inner_pres, SOR_TOL_PRESSURE), then the post-CG corrections with
    ! cfg%alpha_p over the same arrays -- sh%p and the velocities of the phases
    ! in the equation are updated in place (f carries c_loc of them). As the
    ! reference, a NaN cg_res replaces the returned continuity residual.
    ! Serial meshes only.
    subroutine pressure_step_gpu(f, m, alpha_p, max_iter, tol, residual, cg_res, n_iter)
        use mod_types_3d, only: mesh_t
        type(eaf_assembly_fields), intent(in) :: f
        type(mesh_t), intent(in) :: m
        real(c_double), intent(in) :: alpha_p, tol
        integer, intent(in) :: max_iter
        real(c_double), intent(out) :: residual, cg_res
        integer, intent(out) :: n_iter
        integer(c_int) :: st, nit
        if (m%is_parallel) error stop 'pressure_step_gpu: decomposed meshes are not supported'
        call ensure_handle(m%nr, m%ntheta, m%nz)
        st = eaf_pressure_step_f64(handle, f, alpha_p, int(max_iter, c_int), tol, &
                                   residual, cg_res, nit)
        n_iter = int(nit)
        if (st /= EAF_OK .and. st /= EAF_ENONFINITE) error stop 'eaf_pressure_step_f64 failed'
    end subroutine pressure_step_gpu

    ! Same dummies as cg_3d_mpi for DECOMPOSED meshes (m%is_parallel): the
    ! blocks of the eight coefficient arrays and phi are gathered onto rank 0
    ! of m%topo%comm_cart, solved there on the GPU as one global system, and
    ! each rank gets back its block of the solution with every halo cell
    ! inside the domain filled (what cg_3d_mpi's closing halo exchange fills,
    ! src/mod_solver_3d.f90:567); residual and n_iter are broadcast. The
    ! answer is the serial solve's (the parallel reference associates its dot
    ! products per rank). Rank 0 must see a GPU.
    subroutine cg_3d_gpu_mpi(aW, aE, aS, aN, aB, aT, aP, Su, phi, m, &
                             max_iter, tol, residual, n_iter)
        use mpi
        use mod_constants, only: dp
        use mod_types_3d, only: mesh_t
        real(dp), intent(in), contiguous  :: aW(-1:,-1:,-1:), aE(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aS(-1:,-1:,-1:), aN(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aB(-1:,-1:,-1:), aT(-1:,-1:,-1:)
        real(dp), intent(in), contiguous  :: aP(-1:,-1:,-1:), Su(-1:,-1:,-1:)
        real(dp), intent(inout), contiguous :: phi(-1:,-1:,-1:)
        type(mesh_t), intent(in) :: m
        integer, intent(in)      :: max_iter
        real(dp), intent(in)     :: tol
        real(dp), intent(out)    :: residual
        integer, intent(out)     :: n_iter
        integer(c_int) :: grid(3), coords(3), loc(3), start(3), st, nit, p
        integer(c_int), allocatable :: allc(:,:)
        integer(c_long_long) :: np1, nu
        integer :: ierr, nprocs, rank, a, nrg, nthg, nzg
        integer, allocatable :: cnt(:), dsp(:), ucnt(:), udsp(:)
        real(c_double), allocatable :: sbuf(:), gbuf(:), glob(:,:), ubuf(:)
        real(c_double) :: res
        real(c_double) :: outv(2)
        ! global extents (m%nr and friends are the local block in a parallel run)
        nrg = m%topo%nr_global; nthg = m%topo%nth_global; nzg = m%topo%nz_global
        call MPI_Comm_size(m%topo%comm_cart, nprocs, ierr)
        call MPI_Comm_rank(m%topo%comm_cart, rank, ierr)
        grid = [m%topo%npr, m%topo%npth, m%topo%npz]
        coords = m%topo%coords
        loc = [m%topo%iloc, m%topo%jloc, m%topo%kloc]
        start = [m%topo%iglobal_start, m%topo%jglobal_start, m%topo%kglobal_start]
        np1 = eaf_mr_pack_count(grid, coords, loc)
        allocate(sbuf(9 * np1))
        st = eaf_mr_pack(aW, grid, coords, loc, sbuf(0*np1+1:))
        st = eaf_mr_pack(aE, grid, coords, loc, sbuf(1*np1+1:))
        st = eaf_mr_pack(aS, grid, coords, loc, sbuf(2*np1+1:))
        st = eaf_mr_pack(aN, grid, coords, loc, sbuf(3*np1+1:))
        st = eaf_mr_pack(aB, grid, coords, loc, sbuf(4*np1+1:))
        st = eaf_mr_pack(aT, grid, coords, loc, sbuf(5*np1+1:))
        st = eaf_mr_pack(aP, grid, coords, loc, sbuf(6*np1+1:))
        st = eaf_mr_pack(Su, grid, coords, loc, sbuf(7*np1+1:))
        st = eaf_mr_pack(phi, grid, coords, loc, sbuf(8*np1+1:))
        allocate(allc(3, 0:nprocs-1), cnt(0:nprocs-1), dsp(0:nprocs-1))
        allocate(ucnt(0:nprocs-1), udsp(0:nprocs-1))
        call MPI_Gather(coords, 3, MPI_INTEGER, allc, 3, MPI_INTEGER, 0, &
                        m%topo%comm_cart, ierr)
        call MPI_Gather(int(9 * np1), 1, MPI_INTEGER, cnt, 1, MPI_INTEGER, 0, &
                        m%topo%comm_cart, ierr)
        if (rank == 0) then
            dsp(0) = 0
            do p = 1, nprocs - 1
                dsp(p) = dsp(p-1) + cnt(p-1)
            end do
            allocate(gbuf(sum(cnt)))
        else
            allocate(gbuf(1))
        end if
        call MPI_Gatherv(sbuf, int(9 * np1), MPI_DOUBLE_PRECISION, gbuf, cnt, dsp, &
                         MPI_DOUBLE_PRECISION, 0, m%topo%comm_cart, ierr)
        if (rank == 0) then
            allocate(glob((nrg+4)*(nthg+4)*(nzg+4), 9))
            glob = 0.0_c_double
            do p = 0, nprocs - 1
                st = eaf_mr_block(nrg, nthg, nzg, grid, allc(:, p), loc, start)
                np1 = cnt(p) / 9
                do a = 1, 9
                    st = eaf_mr_place(glob(:, a), nrg, nthg, nzg, grid, allc(:, p), loc, &
                                      start, gbuf(dsp(p) + (a-1)*np1 + 1:))
                end do
            end do
            call ensure_handle(nrg, nthg, nzg)
            st = eaf_cg_solve_f64(handle, glob(:,1), glob(:,2), glob(:,3), glob(:,4), &
                                  glob(:,5), glob(:,6), glob(:,7), glob(:,8), glob(:,9), &
                                  int(max_iter, c_int), real(tol, c_double), res, nit)
            if (st /= EAF_OK .and. st /= EAF_ENONFINITE) error stop 'eaf_cg_solve_f64 failed'
            outv = [res, real(nit, c_double)]
            do p = 0, nprocs - 1
                st = eaf_mr_block(nrg, nthg, nzg, grid, allc(:, p), loc, start)
                ucnt(p) = int(eaf_mr_unpack_count(nrg, nzg, start, loc))
            end do
            udsp(0) = 0
            do p = 1, nprocs - 1
                udsp(p) = udsp(p-1) + ucnt(p-1)
            end do
            allocate(ubuf(sum(ucnt)))
            do p = 0, nprocs - 1
                st = eaf_mr_block(nrg, nthg, nzg, grid, allc(:, p), loc, start)
                st = eaf_mr_extract(glob(:, 9), nrg, nthg, nzg, loc, start, ubuf(udsp(p)+1:))
            end do
        else
            allocate(ubuf(1))
        end if
        loc = [m%topo%iloc, m%topo%jloc, m%topo%kloc]
        start = [m%topo%iglobal_start, m%topo%jglobal_start, m%topo%kglobal_start]
        nu = eaf_mr_unpack_count(nrg, nzg, start, loc)
        deallocate(sbuf)
        allocate(sbuf(nu))
        call MPI_Scatterv(ubuf, ucnt, udsp, MPI_DOUBLE_PRECISION, sbuf, int(nu), &
                          MPI_DOUBLE_PRECISION, 0, m%topo%comm_cart, ierr)
        st = eaf_mr_unpack(phi, nrg, nzg, loc, start, sbuf)
        call MPI_Bcast(outv, 2, MPI_DOUBLE_PRECISION, 0, m%topo%comm_cart, ierr)
        residual = outv(1)
        n_iter = int(outv(2))
    end subroutine cg_3d_gpu_mpi

    subroutine cg_gpu_release()
        integer(c_int) :: st
        if (c_associated(handle)) st = eaf_cg_destroy(handle)
        handle = c_null_ptr
        h_nr = -1; h_nth = -1; h_nz = -1
    end subroutine cg_gpu_release

end module mod_solver_gpu
