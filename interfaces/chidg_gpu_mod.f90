!> iso_c_binding interface to the B200 linear-solve library (include/chidg_gpu.h).
!!
!! This module is the Fortran side of the drop-in: ChiDG's containers keep a
!! type(c_ptr) handle (as they keep wrapped_petsc_matrix for backend='petsc',
!! src/containers/type_chidg_matrix.f90:41) and forward init/store/solve calls
!! here when mod_io::backend == 'cuda'.  No Fortran compiler exists in the
!! build environment of this repository, so this file is not compiled here;
!! the same entry points are exercised through ctypes by tests/.
module chidg_gpu_mod
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: CHIDG_GPU_OK = 0, CHIDG_GPU_EINVAL = 1, CHIDG_GPU_ENOMEM = 2,  &
                                 CHIDG_GPU_ESINGULAR = 3, CHIDG_GPU_ENONFINITE = 4,                &
                                 CHIDG_GPU_ETIMEOUT = 5, CHIDG_GPU_ENOTCONVERGED = 6,              &
                                 CHIDG_GPU_ECUDA = 7, CHIDG_GPU_ESTATE = 8
    integer(c_int), parameter :: CHIDG_BLK_LOCAL = 0, CHIDG_BLK_CHIMERA = 1, CHIDG_BLK_BC = 2, CHIDG_BLK_HB = 3
    integer(c_int), parameter :: CHIDG_PRECON_IDENTITY = 0, CHIDG_PRECON_JACOBI = 1, &
                                 CHIDG_PRECON_ILU0 = 2, CHIDG_PRECON_RASILU0 = 3, CHIDG_PRECON_HB = 4
    integer(c_int), parameter :: CHIDG_GPU_FP64 = 0, CHIDG_GPU_MIXED_FP32 = 1, CHIDG_GPU_MIXED_BF16 = 2, &
                                 CHIDG_GPU_MIXED_PRECON_FP32 = 3
    integer(c_int), parameter :: CHIDG_ORTH_CGS = 0, CHIDG_ORTH_MGS = 1
    integer(c_int), parameter :: CHIDG_SCHED_LEVELS = 0, CHIDG_SCHED_DATAFLOW = 1, CHIDG_SCHED_TASKS = 2, &
                                 CHIDG_SCHED_STREAM = 3
    integer(c_int), parameter :: CHIDG_EULER_FARFIELD = 0, CHIDG_EULER_EXTRAPOLATE = 1

    type, bind(c) :: chidg_gpu_pattern
        integer(c_int32_t) :: nelem, ntime
        type(c_ptr)        :: elem_nvars, elem_nterms, elem_proc
        integer(c_int64_t) :: nblocks
        type(c_ptr)        :: blk_row_elem, blk_row_time, blk_col_elem, blk_col_time, blk_kind
    end type chidg_gpu_pattern

    type, bind(c) :: chidg_gpu_fgmres_opts
        real(c_double)     :: tol, rtol
        integer(c_int32_t) :: nmax, nkrylov, orthogonalization, inner_fgmres
        real(c_double)     :: inner_tol, inner_rtol
        integer(c_int32_t) :: inner_nmax, inner_nkrylov, inner_orthogonalization
        integer(c_int32_t) :: use_controller, precision, mixed_inner_nkrylov
        real(c_double)     :: mixed_inner_rtol
        integer(c_int32_t) :: mixed_inner_nmax
    end type chidg_gpu_fgmres_opts

    ! chidg_gpu_euler_box: the Euler box of chidg_gpu_euler_create
    type, bind(c) :: chidg_gpu_euler_box
        integer(c_int32_t) :: nx, ny, nz, order
        real(c_double)     :: lo(3), hi(3)
        integer(c_int32_t) :: bc(6)
        real(c_double)     :: rho_inf, p_inf
        real(c_double)     :: vel_inf(3)
    end type chidg_gpu_euler_box

    ! chidg_gpu_euler_system: a Newton system of chidg_gpu_euler_fill_system
    type, bind(c) :: chidg_gpu_euler_system
        type(chidg_gpu_euler_box) :: box
        integer(c_int32_t)        :: ntime
        type(c_ptr)               :: level_vel, D, mass, q0
        real(c_double)            :: cfl
    end type chidg_gpu_euler_system

    type, bind(c) :: chidg_gpu_fgmres_result
        integer(c_int32_t) :: niter, nrestart, inner_iters, nhist
        real(c_double)     :: residual_norm, res_estimate, r0norm_initial, seconds
    end type chidg_gpu_fgmres_result

    interface
        integer(c_int) function chidg_gpu_ctx_create(device, stream, ctx) bind(c, name='chidg_gpu_ctx_create')
            import :: c_int, c_ptr
            integer(c_int), value :: device
            type(c_ptr),    value :: stream
            type(c_ptr)           :: ctx
        end function
        integer(c_int) function chidg_gpu_ctx_destroy(ctx) bind(c, name='chidg_gpu_ctx_destroy')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function
        integer(c_int) function chidg_gpu_last_error(ctx, buf, buflen) bind(c, name='chidg_gpu_last_error')
            import :: c_int, c_ptr, c_char, c_int32_t
            type(c_ptr), value        :: ctx
            character(kind=c_char)    :: buf(*)
            integer(c_int32_t), value :: buflen
        end function
        integer(c_int) function chidg_gpu_error_element(ctx, elem) bind(c, name='chidg_gpu_error_element')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: ctx
            integer(c_int32_t) :: elem
        end function
        integer(c_int) function chidg_gpu_matrix_create(ctx, pat, mat) bind(c, name='chidg_gpu_matrix_create')
            import :: c_int, c_ptr, chidg_gpu_pattern
            type(c_ptr), value      :: ctx
            type(chidg_gpu_pattern) :: pat
            type(c_ptr)             :: mat
        end function
        integer(c_int) function chidg_gpu_matrix_destroy(mat) bind(c, name='chidg_gpu_matrix_destroy')
            import :: c_int, c_ptr
            type(c_ptr), value :: mat
        end function
        integer(c_int) function chidg_gpu_matrix_upload_blocks(mat, ptrs) bind(c, name='chidg_gpu_matrix_upload_blocks')
            import :: c_int, c_ptr
            type(c_ptr), value :: mat
            type(c_ptr)        :: ptrs(*)
        end function
        integer(c_int) function chidg_gpu_matrix_upload(mat, vals) bind(c, name='chidg_gpu_matrix_upload')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: mat
            real(c_double)     :: vals(*)
        end function
        integer(c_int) function chidg_gpu_matrix_clear(mat) bind(c, name='chidg_gpu_matrix_clear')
            import :: c_int, c_ptr
            type(c_ptr), value :: mat
        end function
        integer(c_int) function chidg_gpu_matrix_scale_diagonal(mat, mass, scale) bind(c, name='chidg_gpu_matrix_scale_diagonal')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: mat
            real(c_double)     :: mass(*), scale(*)
        end function
        ! chidg_matrix_t%transposed (type_chidg_matrix.f90:49)
        integer(c_int) function chidg_gpu_matrix_set_transposed(mat, transposed) bind(c, name='chidg_gpu_matrix_set_transposed')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: mat
            integer(c_int32_t), value :: transposed
        end function
        integer(c_int) function chidg_gpu_matrix_get_transposed(mat, transposed) bind(c, name='chidg_gpu_matrix_get_transposed')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: mat
            integer(c_int32_t) :: transposed
        end function
        ! chidg_matrix%to_file (type_chidg_matrix.f90:1451-1507); path NUL-terminated
        integer(c_int) function chidg_gpu_matrix_to_file(mat, path) bind(c, name='chidg_gpu_matrix_to_file')
            import :: c_int, c_ptr, c_char
            type(c_ptr), value     :: mat
            character(kind=c_char) :: path(*)
        end function
        integer(c_int) function chidg_gpu_matrix_save(mat, path) bind(c, name='chidg_gpu_matrix_save')
            import :: c_int, c_ptr, c_char
            type(c_ptr), value     :: mat
            character(kind=c_char) :: path(*)
        end function
        integer(c_int) function chidg_gpu_matrix_load(ctx, path, mat) bind(c, name='chidg_gpu_matrix_load')
            import :: c_int, c_ptr, c_char
            type(c_ptr), value     :: ctx
            character(kind=c_char) :: path(*)
            type(c_ptr)            :: mat
        end function
        integer(c_int) function chidg_gpu_vector_create(mat, vec) bind(c, name='chidg_gpu_vector_create')
            import :: c_int, c_ptr
            type(c_ptr), value :: mat
            type(c_ptr)        :: vec
        end function
        integer(c_int) function chidg_gpu_vector_destroy(vec) bind(c, name='chidg_gpu_vector_destroy')
            import :: c_int, c_ptr
            type(c_ptr), value :: vec
        end function
        integer(c_int) function chidg_gpu_vector_upload(vec, vals) bind(c, name='chidg_gpu_vector_upload')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: vec
            real(c_double)     :: vals(*)
        end function
        integer(c_int) function chidg_gpu_vector_download(vec, vals) bind(c, name='chidg_gpu_vector_download')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: vec
            real(c_double)     :: vals(*)
        end function
        integer(c_int) function chidg_gpu_matvec(mat, x, y) bind(c, name='chidg_gpu_matvec')
            import :: c_int, c_ptr
            type(c_ptr), value :: mat, x, y
        end function
        ! chidg_vector%norm_fields (type_chidg_vector.f90:1319-1352)
        integer(c_int) function chidg_gpu_vector_norm_fields(x, nrm, nfields) bind(c, name='chidg_gpu_vector_norm_fields')
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr),        value :: x
            real(c_double)            :: nrm(*)
            integer(c_int32_t), value :: nfields
        end function
        integer(c_int) function chidg_gpu_vector_norm(x, nrm) bind(c, name='chidg_gpu_vector_norm')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: x
            real(c_double)     :: nrm
        end function
        integer(c_int) function chidg_gpu_precon_create(mat, kind, M) bind(c, name='chidg_gpu_precon_create')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value        :: mat
            integer(c_int32_t), value :: kind
            type(c_ptr)               :: M
        end function
        integer(c_int) function chidg_gpu_precon_update(M, mat, precision) bind(c, name='chidg_gpu_precon_update')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value        :: M, mat
            integer(c_int32_t), value :: precision
        end function
        integer(c_int) function chidg_gpu_precon_apply(M, mat, v, z) bind(c, name='chidg_gpu_precon_apply')
            import :: c_int, c_ptr
            type(c_ptr), value :: M, mat, v, z
        end function
        integer(c_int) function chidg_gpu_precon_destroy(M) bind(c, name='chidg_gpu_precon_destroy')
            import :: c_int, c_ptr
            type(c_ptr), value :: M
        end function
        integer(c_int) function chidg_gpu_fgmres_solve(mat, M, b, x, opts, res, hist, hist_cap) &
                bind(c, name='chidg_gpu_fgmres_solve')
            import :: c_int, c_ptr, c_double, c_int32_t, chidg_gpu_fgmres_opts, chidg_gpu_fgmres_result
            type(c_ptr), value            :: mat, M, b, x
            type(chidg_gpu_fgmres_opts)   :: opts
            type(chidg_gpu_fgmres_result) :: res
            real(c_double)                :: hist(*)
            integer(c_int32_t), value     :: hist_cap
        end function
        integer(c_int) function chidg_gpu_fgmres_default_opts(opts) bind(c, name='chidg_gpu_fgmres_default_opts')
            import :: c_int, chidg_gpu_fgmres_opts
            type(chidg_gpu_fgmres_opts) :: opts
        end function
        integer(c_int) function chidg_gpu_euler_create(ctx, box, E) bind(c, name='chidg_gpu_euler_create')
            import :: c_int, c_ptr, chidg_gpu_euler_box
            type(c_ptr), value        :: ctx
            type(chidg_gpu_euler_box) :: box
            type(c_ptr)               :: E
        end function
        integer(c_int) function chidg_gpu_euler_destroy(E) bind(c, name='chidg_gpu_euler_destroy')
            import :: c_int, c_ptr
            type(c_ptr), value :: E
        end function
        ! pass c_null_ptr as mat for the residual alone (the line search)
        integer(c_int) function chidg_gpu_euler_assemble(E, q, rhs, mat) bind(c, name='chidg_gpu_euler_assemble')
            import :: c_int, c_ptr
            type(c_ptr), value :: E, q, rhs, mat
        end function
        integer(c_int) function chidg_gpu_euler_pseudo_timestep(E, q, cfl, dtau) &
                bind(c, name='chidg_gpu_euler_pseudo_timestep')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: E, q
            real(c_double)     :: cfl(5), dtau(*)
        end function
        ! ---- context utilities --------------------------------------------
        integer(c_int) function chidg_gpu_ctx_sync(ctx) bind(c, name='chidg_gpu_ctx_sync')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
        end function
        integer(c_int) function chidg_gpu_launch_count(ctx, count) bind(c, name='chidg_gpu_launch_count')
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: ctx
            integer(c_int64_t) :: count
        end function
        integer(c_int) function chidg_gpu_ctx_set_profiling(ctx, on) bind(c, name='chidg_gpu_ctx_set_profiling')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: ctx
            integer(c_int32_t), value :: on
        end function
        integer(c_int) function chidg_gpu_ctx_kernel_time(ctx, kernel_class, total_ms, count) &
                bind(c, name='chidg_gpu_ctx_kernel_time')
            import :: c_int, c_ptr, c_int32_t, c_int64_t, c_double
            type(c_ptr),        value :: ctx
            integer(c_int32_t), value :: kernel_class
            real(c_double)            :: total_ms
            integer(c_int64_t)        :: count
        end function
        integer(c_int) function chidg_gpu_host_alloc(bytes, p) bind(c, name='chidg_gpu_host_alloc')
            import :: c_int, c_ptr, c_size_t
            integer(c_size_t), value :: bytes
            type(c_ptr)              :: p
        end function
        integer(c_int) function chidg_gpu_host_free(p) bind(c, name='chidg_gpu_host_free')
            import :: c_int, c_ptr
            type(c_ptr), value :: p
        end function
        integer(c_int) function chidg_gpu_selftest_bounded_waits(ctx, limit_cycles, bits) &
                bind(c, name='chidg_gpu_selftest_bounded_waits')
            import :: c_int, c_ptr, c_int32_t, c_int64_t
            type(c_ptr),        value :: ctx
            integer(c_int64_t), value :: limit_cycles
            integer(c_int32_t)        :: bits
        end function
        ! ---- chidg_matrix_t accessors and partial stores --------------------
        integer(c_int) function chidg_gpu_matrix_nvalues(mat, nvalues) bind(c, name='chidg_gpu_matrix_nvalues')
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: mat
            integer(c_int64_t) :: nvalues
        end function
        integer(c_int) function chidg_gpu_matrix_nvec(mat, n) bind(c, name='chidg_gpu_matrix_nvec')
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: mat
            integer(c_int64_t) :: n
        end function
        ! values already on the device (a device pointer passed by value)
        integer(c_int) function chidg_gpu_matrix_upload_device(mat, dev) bind(c, name='chidg_gpu_matrix_upload_device')
            import :: c_int, c_ptr
            type(c_ptr), value :: mat, dev
        end function
        ! chidg_matrix%store of a range of the packed values (bumps the stamp)
        integer(c_int) function chidg_gpu_matrix_upload_range(mat, vals, first, count) &
                bind(c, name='chidg_gpu_matrix_upload_range')
            import :: c_int, c_ptr, c_double, c_int64_t
            type(c_ptr),        value :: mat
            real(c_double)            :: vals(*)
            integer(c_int64_t), value :: first, count
        end function
        integer(c_int) function chidg_gpu_matrix_download(mat, vals) bind(c, name='chidg_gpu_matrix_download')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: mat
            real(c_double)     :: vals(*)
        end function
        ! chidg_matrix_t%stamp (type_chidg_matrix.f90:575-747): a counter bumped by every store
        integer(c_int) function chidg_gpu_matrix_stamp(mat, stamp) bind(c, name='chidg_gpu_matrix_stamp')
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: mat
            integer(c_int64_t) :: stamp
        end function
        integer(c_int) function chidg_gpu_matrix_get_pattern(mat, nelem, ntime, nblocks, elem_nvars, elem_nterms, &
                elem_proc, blk_row_elem, blk_row_time, blk_col_elem, blk_col_time, blk_kind) &
                bind(c, name='chidg_gpu_matrix_get_pattern')
            import :: c_int, c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: mat
            integer(c_int32_t) :: nelem, ntime
            integer(c_int64_t) :: nblocks
            integer(c_int32_t) :: elem_nvars(*), elem_nterms(*), elem_proc(*)
            integer(c_int32_t) :: blk_row_elem(*), blk_row_time(*), blk_col_elem(*), blk_col_time(*), blk_kind(*)
        end function
        ! ---- chidg_vector_t operators (type_chidg_vector.f90) ----------------
        integer(c_int) function chidg_gpu_vector_upload_range(vec, vals, first, count) &
                bind(c, name='chidg_gpu_vector_upload_range')
            import :: c_int, c_ptr, c_double, c_int64_t
            type(c_ptr),        value :: vec
            real(c_double)            :: vals(*)
            integer(c_int64_t), value :: first, count
        end function
        integer(c_int) function chidg_gpu_vector_upload_device(vec, dev) bind(c, name='chidg_gpu_vector_upload_device')
            import :: c_int, c_ptr
            type(c_ptr), value :: vec, dev
        end function
        integer(c_int) function chidg_gpu_vector_device_ptr(vec, dev) bind(c, name='chidg_gpu_vector_device_ptr')
            import :: c_int, c_ptr
            type(c_ptr), value :: vec
            type(c_ptr)        :: dev
        end function
        integer(c_int) function chidg_gpu_vector_clear(vec) bind(c, name='chidg_gpu_vector_clear')
            import :: c_int, c_ptr
            type(c_ptr), value :: vec
        end function
        integer(c_int) function chidg_gpu_vector_copy(dst, src) bind(c, name='chidg_gpu_vector_copy')
            import :: c_int, c_ptr
            type(c_ptr), value :: dst, src
        end function
        ! y = y + a x
        integer(c_int) function chidg_gpu_vector_axpy(y, a, x) bind(c, name='chidg_gpu_vector_axpy')
            import :: c_int, c_ptr, c_double
            type(c_ptr),    value :: y
            real(c_double), value :: a
            type(c_ptr),    value :: x
        end function
        integer(c_int) function chidg_gpu_vector_scale(x, a) bind(c, name='chidg_gpu_vector_scale')
            import :: c_int, c_ptr, c_double
            type(c_ptr),    value :: x
            real(c_double), value :: a
        end function
        integer(c_int) function chidg_gpu_vector_mass_scale(x, y, mass, scale) bind(c, name='chidg_gpu_vector_mass_scale')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: x, y
            real(c_double)     :: mass(*), scale(*)
        end function
        ! dot (operator_chidg_dot.f90:30-97)
        integer(c_int) function chidg_gpu_vector_dot(x, y, res) bind(c, name='chidg_gpu_vector_dot')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: x, y
            real(c_double)     :: res
        end function
        ! dot of two device arrays with no device allocation (no counterpart in the reference)
        integer(c_int) function chidg_gpu_dot_noalloc(device, x, y, n, res, stream) bind(c, name='chidg_gpu_dot_noalloc')
            import :: c_int, c_ptr, c_int64_t
            integer(c_int),     value :: device
            type(c_ptr),        value :: x, y
            integer(c_int64_t), value :: n
            type(c_ptr),        value :: res, stream
        end function
        ! ---- preconditioner_t extras -----------------------------------------
        integer(c_int) function chidg_gpu_precon_set_schedule(M, schedule) bind(c, name='chidg_gpu_precon_set_schedule')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: M
            integer(c_int32_t), value :: schedule
        end function
        integer(c_int) function chidg_gpu_precon_download_LD(M, vals) bind(c, name='chidg_gpu_precon_download_LD')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: M
            real(c_double)     :: vals(*)
        end function
        integer(c_int) function chidg_gpu_precon_download_LD32(M, vals) bind(c, name='chidg_gpu_precon_download_LD32')
            import :: c_int, c_ptr, c_float
            type(c_ptr), value :: M
            real(c_float)      :: vals(*)
        end function
        ! preconditioner_t%stamp (type_preconditioner.f90:21-121)
        integer(c_int) function chidg_gpu_precon_stamp(M, stamp) bind(c, name='chidg_gpu_precon_stamp')
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: M
            integer(c_int64_t) :: stamp
        end function
        ! ---- many independent systems in one call ------------------------------
        integer(c_int) function chidg_gpu_fgmres_solve_batched(mat, M, nsys, sys_elem, b, x, opts, results, hist, &
                hist_cap) bind(c, name='chidg_gpu_fgmres_solve_batched')
            import :: c_int, c_ptr, c_double, c_int32_t, chidg_gpu_fgmres_opts, chidg_gpu_fgmres_result
            type(c_ptr),        value     :: mat, M
            integer(c_int32_t), value     :: nsys
            integer(c_int32_t)            :: sys_elem(*)
            type(c_ptr),        value     :: b, x
            type(chidg_gpu_fgmres_opts)   :: opts
            type(chidg_gpu_fgmres_result) :: results(*)
            real(c_double)                :: hist(*)
            integer(c_int32_t), value     :: hist_cap
        end function
        ! the Euler box at elements elem0.. of a larger layout (a batch arena)
        integer(c_int) function chidg_gpu_euler_assemble_at(E, mat, elem0, q, rhs, jacobian) &
                bind(c, name='chidg_gpu_euler_assemble_at')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: E, mat
            integer(c_int32_t), value :: elem0
            type(c_ptr),        value :: q, rhs
            integer(c_int32_t), value :: jacobian
        end function
        integer(c_int) function chidg_gpu_euler_pseudo_timestep_at(E, mat, elem0, q, cfl, dtau) &
                bind(c, name='chidg_gpu_euler_pseudo_timestep_at')
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr),        value :: E, mat
            integer(c_int32_t), value :: elem0
            type(c_ptr),        value :: q
            real(c_double)            :: cfl(5), dtau(*)
        end function
        ! harmonic balance: one level's spatial part, that level's dtau, the time coupling
        integer(c_int) function chidg_gpu_euler_assemble_level(E, mat, itime, q, rhs, jacobian) &
                bind(c, name='chidg_gpu_euler_assemble_level')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: E, mat
            integer(c_int32_t), value :: itime
            type(c_ptr),        value :: q, rhs
            integer(c_int32_t), value :: jacobian
        end function
        integer(c_int) function chidg_gpu_euler_pseudo_timestep_level(E, mat, itime, q, cfl, dtau) &
                bind(c, name='chidg_gpu_euler_pseudo_timestep_level')
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr),        value :: E, mat
            integer(c_int32_t), value :: itime
            type(c_ptr),        value :: q
            real(c_double)            :: cfl(5), dtau(*)
        end function
        integer(c_int) function chidg_gpu_hb_coupling(mat, nterms, D, mass, q, rhs, jacobian) &
                bind(c, name='chidg_gpu_hb_coupling')
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr),        value :: mat
            integer(c_int32_t), value :: nterms
            real(c_double)            :: D(*), mass(*)
            type(c_ptr),        value :: q, rhs
            integer(c_int32_t), value :: jacobian
        end function
        integer(c_int) function chidg_gpu_euler_assemble_level_at(E, mat, elem0, itime, q, rhs, jacobian) &
                bind(c, name='chidg_gpu_euler_assemble_level_at')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: E, mat
            integer(c_int32_t), value :: elem0, itime
            type(c_ptr),        value :: q, rhs
            integer(c_int32_t), value :: jacobian
        end function
        integer(c_int) function chidg_gpu_hb_coupling_at(mat, elem0, nelem, nterms, D, mass, q, rhs, jacobian) &
                bind(c, name='chidg_gpu_hb_coupling_at')
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr),        value :: mat
            integer(c_int32_t), value :: elem0, nelem, nterms
            real(c_double)            :: D(*), mass(*)
            type(c_ptr),        value :: q, rhs
            integer(c_int32_t), value :: jacobian
        end function
        ! pass c_null_ptr as rhs to leave the right-hand side as it is
        integer(c_int) function chidg_gpu_euler_pseudo_transient_at(E, mat, elem0, q, rhs, cfl, mass) &
                bind(c, name='chidg_gpu_euler_pseudo_transient_at')
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr),        value :: E, mat
            integer(c_int32_t), value :: elem0
            type(c_ptr),        value :: q, rhs
            real(c_double)            :: cfl(5), mass(*)
        end function
        ! user: c_loc of a chidg_gpu_euler_system; also usable as a chidg_gpu_fill_fn
        ! (c_funloc(chidg_gpu_euler_fill_system)) for chidg_gpu_serve_submit_fill
        integer(c_int) function chidg_gpu_euler_fill_system(user, ctx, mat, b, work, elem0) &
                bind(c, name='chidg_gpu_euler_fill_system')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: user, ctx, mat, b, work
            integer(c_int32_t), value :: elem0
        end function
        ! ---- launch shapes of the streamed kernels and their autotuner --------
        integer(c_int) function chidg_gpu_autotune(M, mat, precision, reps) bind(c, name='chidg_gpu_autotune')
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr),        value :: M, mat
            integer(c_int32_t), value :: precision, reps
        end function
        integer(c_int) function chidg_gpu_stream_shape_get(kind, max_b, value_bytes, warps, stages, stage_bytes) &
                bind(c, name='chidg_gpu_stream_shape_get')
            import :: c_int, c_int32_t
            integer(c_int32_t), value :: kind, max_b, value_bytes
            integer(c_int32_t)        :: warps, stages, stage_bytes
        end function
        integer(c_int) function chidg_gpu_stream_shape_set(kind, max_b, value_bytes, warps, stages, stage_bytes) &
                bind(c, name='chidg_gpu_stream_shape_set')
            import :: c_int, c_int32_t
            integer(c_int32_t), value :: kind, max_b, value_bytes, warps, stages, stage_bytes
        end function
        ! ---- request server ----------------------------------------------------
        integer(c_int) function chidg_gpu_serve_create(device, slots, mem_budget, max_batch, precon_kind, opts, srv) &
                bind(c, name='chidg_gpu_serve_create')
            import :: c_int, c_ptr, c_int32_t, c_int64_t, chidg_gpu_fgmres_opts
            integer(c_int),     value   :: device
            integer(c_int32_t), value   :: slots
            integer(c_int64_t), value   :: mem_budget
            integer(c_int32_t), value   :: max_batch, precon_kind
            type(chidg_gpu_fgmres_opts) :: opts
            type(c_ptr)                 :: srv
        end function
        integer(c_int) function chidg_gpu_serve_submit(srv, pat, vals, rhs, ticket) bind(c, name='chidg_gpu_serve_submit')
            import :: c_int, c_ptr, c_double, c_int64_t, chidg_gpu_pattern
            type(c_ptr), value      :: srv
            type(chidg_gpu_pattern) :: pat
            real(c_double)          :: vals(*), rhs(*)
            integer(c_int64_t)      :: ticket
        end function
        integer(c_int) function chidg_gpu_serve_wait(srv, ticket, x, res, timing) bind(c, name='chidg_gpu_serve_wait')
            import :: c_int, c_ptr, c_double, c_int64_t, chidg_gpu_fgmres_result
            type(c_ptr),        value     :: srv
            integer(c_int64_t), value     :: ticket
            real(c_double)                :: x(*)
            type(chidg_gpu_fgmres_result) :: res
            real(c_double)                :: timing(*)
        end function
        integer(c_int) function chidg_gpu_serve_stats(srv, batches, peak_mem_bytes) bind(c, name='chidg_gpu_serve_stats')
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: srv
            integer(c_int64_t) :: batches, peak_mem_bytes
        end function
        integer(c_int) function chidg_gpu_serve_destroy(srv) bind(c, name='chidg_gpu_serve_destroy')
            import :: c_int, c_ptr
            type(c_ptr), value :: srv
        end function
        ! fill: c_funloc of a function with chidg_gpu_fill_fn's interface; user stays
        ! valid until the request's wait returns
        integer(c_int) function chidg_gpu_serve_submit_fill(srv, pat, fill, user, ticket) &
                bind(c, name='chidg_gpu_serve_submit_fill')
            import :: c_int, c_ptr, c_funptr, c_int64_t, chidg_gpu_pattern
            type(c_ptr),    value   :: srv
            type(chidg_gpu_pattern) :: pat
            type(c_funptr), value   :: fill
            type(c_ptr),    value   :: user
            integer(c_int64_t)      :: ticket
        end function
        integer(c_int) function chidg_gpu_serve_batch_log(srv, i, rec) bind(c, name='chidg_gpu_serve_batch_log')
            import :: c_int, c_ptr, c_int64_t, c_double
            type(c_ptr),        value :: srv
            integer(c_int64_t), value :: i
            real(c_double)            :: rec(9)
        end function
    end interface

end module chidg_gpu_mod
