!! pned_gpu.f90 -- iso_c_binding interface to libpned_gpu.so for pNED's
!! Fortran host.  With this module a solver file switches its H.v from the
!! MPI/OpenMP p_mltply_v3 to the GPU by `use pned_gpu` and calling
!! p_mltply_v3_gpu with the same arguments (S_one_half/Hybrid_TPS_parallel.f90:190).
!! Not compiled in the build container (no Fortran compiler there).
module pned_gpu
  use iso_c_binding
  implicit none
  private
  public :: pned_gpu_init, pned_gpu_finalize, p_mltply_v3_gpu, calc_vec_inprdct_gpu, pned_lanczos_run_f
  public :: pned_lncv1_f, pned_inv1_f, pned_tps_run_f, pned_dump_alpha_beta_coef_f
  public :: pned_lanczos_begin_f, pned_steps_f, pned_lanczos_read_f, pned_interval_dump_f, pned_interval_dump_read_f
  public :: pned_gpu_init_target, pned_dsf_zz_f, pned_dsf_xy_f, pned_append_sq_f, pned_dump_alpha_beta_f
  public :: pned_lanczos_state_f, pned_lanczos_resume_f

  type, bind(C) :: pned_model_desc
    integer(c_int32_t) :: n_sites, q_spin, tree, n_bonds
    type(c_ptr) :: ipair, bond_type, xlocal, skip
    integer(c_int32_t) :: parity_type, total_sz
  end type pned_model_desc

  interface
    integer(c_int) function pned_model_create(desc, m) bind(C, name="pned_model_create")
      import :: pned_model_desc, c_int, c_ptr
      type(pned_model_desc), intent(in) :: desc
      type(c_ptr), intent(out) :: m
    end function
    integer(c_int) function pned_ctx_create(m, R, budget, c) bind(C, name="pned_ctx_create")
      import :: c_int, c_ptr, c_size_t
      type(c_ptr), value :: m
      integer(c_int), value :: R
      integer(c_size_t), value :: budget
      type(c_ptr), intent(out) :: c
    end function
    integer(c_int) function pned_hv(c, v1, v0, eperbd, prdct, flags) bind(C, name="pned_hv")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c
      complex(c_double_complex), intent(in) :: v1(*)
      complex(c_double_complex), intent(inout) :: v0(*)
      real(c_double), value :: eperbd
      complex(c_double_complex), intent(out) :: prdct
      integer(c_int), value :: flags
    end function
    integer(c_int) function pned_inprdct(c, x1, x2, out, flags) bind(C, name="pned_inprdct")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: c
      complex(c_double_complex), intent(in) :: x1(*), x2(*)
      complex(c_double_complex), intent(out) :: out
      integer(c_int), value :: flags
    end function
    integer(c_int) function pned_lanczos_run(c, v, nsteps, check_conv, alpha, beta, ene, done, flags) &
        bind(C, name="pned_lanczos_run")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c
      complex(c_double_complex), intent(in) :: v(*)
      integer(c_int), value :: nsteps, check_conv, flags
      real(c_double), intent(out) :: alpha(*), beta(*), ene(8)
      integer(c_int), intent(out) :: done
    end function
    integer(c_int) function pned_lanczos_vector(c, v, nsteps, alpha, beta, coef, x, flags) &
        bind(C, name="pned_lanczos_vector")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c
      complex(c_double_complex), intent(in) :: v(*)
      integer(c_int), value :: nsteps, flags
      real(c_double), intent(in) :: alpha(*), beta(*), coef(*)
      complex(c_double_complex), intent(out) :: x(*)
    end function
    integer(c_int) function pned_cg_run(c, e, b, inv_max, cg_max, x, n_inv, n_cg, flags) bind(C, name="pned_cg_run")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c
      real(c_double), value :: e
      complex(c_double_complex), intent(in) :: b(*)
      integer(c_int), value :: inv_max, cg_max, flags
      complex(c_double_complex), intent(out) :: x(*)
      integer(c_int), intent(out) :: n_inv, n_cg
    end function
    integer(c_int) function pned_tps_run(c, L, v, nsteps, nobs, obs, alpha, beta, coef, flags) &
        bind(C, name="pned_tps_run")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c, obs
      real(c_double), value :: L
      complex(c_double_complex), intent(in) :: v(*)
      integer(c_int), value :: nsteps, nobs, flags
      real(c_double), intent(out) :: alpha(*), beta(*), coef(*)
    end function
    integer(c_int) function pned_write_salphasbeta(path, n1, n2, alpha, beta, coef) &
        bind(C, name="pned_write_salphasbeta")
      import :: c_int, c_char, c_double
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), value :: n1, n2
      real(c_double), intent(in) :: alpha(*), beta(*), coef(*)
    end function
    integer(c_int) function pned_session_begin(c, kind, v, max_steps, L, nobs, obs, flags) &
        bind(C, name="pned_session_begin")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c, obs
      integer(c_int), value :: kind, max_steps, nobs, flags
      complex(c_double_complex), intent(in) :: v(*)
      real(c_double), value :: L
    end function
    integer(c_int) function pned_session_step(c, nsteps) bind(C, name="pned_session_step")
      import :: c_int, c_ptr
      type(c_ptr), value :: c
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function pned_session_read(c, alpha, beta, coef, done, status) bind(C, name="pned_session_read")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: c, coef
      real(c_double), intent(out) :: alpha(*), beta(*)
      integer(c_int), intent(out) :: done, status
    end function
    integer(c_int) function pned_session_save(c, path) bind(C, name="pned_session_save")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: c
      character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function pned_session_load(c, path, max_steps) bind(C, name="pned_session_load")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: c
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), value :: max_steps
    end function
    integer(c_int) function pned_session_lanczos_state(c, w, v, flags) bind(C, name="pned_session_lanczos_state")
      import :: c_int, c_ptr, c_double_complex
      type(c_ptr), value :: c
      complex(c_double_complex), intent(out) :: w(*), v(*)
      integer(c_int), value :: flags
    end function
    integer(c_int) function pned_session_begin_lanczos_at(c, w, v, alpha, beta, k, max_steps, flags) &
        bind(C, name="pned_session_begin_lanczos_at")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c
      complex(c_double_complex), intent(in) :: w(*), v(*)
      real(c_double), intent(in) :: alpha(*), beta(*)
      integer(c_int), value :: k, max_steps, flags
    end function
    integer(c_int) function pned_dsf_run(c, x, qr, nsteps, cnorm, salpha, sbeta, flags) bind(C, name="pned_dsf_run")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c
      complex(c_double_complex), intent(in) :: x(*)
      real(c_double), intent(in) :: qr(*)
      integer(c_int), value :: nsteps, flags
      real(c_double), intent(out) :: cnorm(*), salpha(*), sbeta(*)
    end function
    integer(c_int) function pned_dsf_xy_run(c, source, ipm, x, qr, nsteps, cnorm, salpha, sbeta, flags) &
        bind(C, name="pned_dsf_xy_run")
      import :: c_int, c_ptr, c_double, c_double_complex
      type(c_ptr), value :: c, source
      integer(c_int), value :: ipm, nsteps, flags
      complex(c_double_complex), intent(in) :: x(*)
      real(c_double), intent(in) :: qr(*)
      real(c_double), intent(out) :: cnorm(*), salpha(*), sbeta(*)
    end function
    integer(c_int) function pned_append_sq(path, iq, q1, q2, norm_re) bind(C, name="pned_append_sq")
      import :: c_int, c_char, c_double
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), value :: iq
      real(c_double), value :: q1, q2, norm_re
    end function
    integer(c_int) function pned_write_dsf_alpha_beta(path, sq, salpha, sbeta, s_maxitr) &
        bind(C, name="pned_write_dsf_alpha_beta")
      import :: c_int, c_char, c_double, c_double_complex
      character(kind=c_char), intent(in) :: path(*)
      complex(c_double_complex), value :: sq
      real(c_double), intent(in) :: salpha(*), sbeta(*)
      integer(c_int), value :: s_maxitr
    end function
    integer(c_int) function pned_write_dsf_vectors(path, indx, v1, v2, ll) bind(C, name="pned_write_dsf_vectors")
      import :: c_int, c_char, c_double_complex, c_int64_t
      character(kind=c_char), intent(in) :: path(*)
      integer(c_int), value :: indx
      complex(c_double_complex), intent(in) :: v1(*), v2(*)
      integer(c_int64_t), value :: ll
    end function
    integer(c_int) function pned_ctx_destroy(c) bind(C, name="pned_ctx_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: c
    end function
    integer(c_int) function pned_model_destroy(m) bind(C, name="pned_model_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: m
    end function
  end interface

  type(c_ptr), save :: g_model = c_null_ptr, g_ctx = c_null_ptr
  !! second model and context: the neighbouring Sz sector of the S^+-_q DSF chains
  type(c_ptr), save :: g_model2 = c_null_ptr, g_ctx2 = c_null_ptr
  integer(c_int32_t), allocatable, target, save :: g_ipair(:), g_btype(:)
  integer(c_int8_t), allocatable, target, save :: g_skip(:,:,:)
  complex(c_double_complex), allocatable, target, save :: g_x(:,:,:)

contains

  !! Builds the device model from the module state of params.f90
  !! (ipair, ibond_type, xlocal_Ham, llocal_Ham, parity_type, total_sz).
  subroutine pned_gpu_init(n, q_spin, tree, ibond, ipair, ibond_type, xlocal_ham, llocal_ham, parity_type, total_sz)
    integer, intent(in) :: n, q_spin, tree, ibond, parity_type, total_sz
    integer, intent(in) :: ipair(2*ibond), ibond_type(ibond)
    complex(kind(0d0)), intent(in) :: xlocal_ham(0:q_spin**2-1, 0:q_spin**2-1, 9)
    logical, intent(in) :: llocal_ham(0:q_spin**2-1, 0:q_spin**2-1, 9)
    type(pned_model_desc) :: d
    integer(c_int) :: rc
    allocate(g_ipair(2*ibond), g_btype(ibond))
    allocate(g_x(0:q_spin**2-1, 0:q_spin**2-1, 9), g_skip(0:q_spin**2-1, 0:q_spin**2-1, 9))
    g_ipair = ipair; g_btype = ibond_type; g_x = xlocal_ham
    g_skip = 0
    where (llocal_ham) g_skip = 1
    d%n_sites = n; d%q_spin = q_spin; d%tree = tree; d%n_bonds = ibond
    d%ipair = c_loc(g_ipair); d%bond_type = c_loc(g_btype)
    d%xlocal = c_loc(g_x); d%skip = c_loc(g_skip)
    d%parity_type = parity_type; d%total_sz = total_sz
    rc = pned_model_create(d, g_model)
    if (rc /= 0) stop 'pned_model_create failed'
    rc = pned_ctx_create(g_model, 1_c_int, 0_c_size_t, g_ctx)
    if (rc /= 0) stop 'pned_ctx_create failed'
  end subroutine pned_gpu_init

  !! Same arguments and meaning as p_mltply_v3: v0 = v0 + (H - eperbd*ibond)^T v1, prdct = <v1|H v1>.
  subroutine p_mltply_v3_gpu(v1, v0, prdct, eperbd)
    complex(kind(0d0)), intent(inout) :: v1(:), v0(:)
    complex(kind(0d0)), intent(inout) :: prdct
    double precision, intent(in) :: eperbd
    integer(c_int) :: rc
    rc = pned_hv(g_ctx, v1, v0, real(eperbd, c_double), prdct, 0_c_int)
    if (rc /= 0) stop 'pned_hv failed'
  end subroutine p_mltply_v3_gpu

  subroutine calc_vec_inprdct_gpu(x1, x2, norm)
    complex(kind(0d0)), intent(in) :: x1(:), x2(:)
    complex(kind(0d0)), intent(inout) :: norm
    integer(c_int) :: rc
    rc = pned_inprdct(g_ctx, x1, x2, norm, 0_c_int)
    if (rc /= 0) stop 'pned_inprdct failed'
  end subroutine calc_vec_inprdct_gpu

  !! Whole parallelized_lnc1z loop on the GPU (alpha/beta as the reference stores them).
  subroutine pned_lanczos_run_f(v, nsteps, check_conv, alpha, beta, ene, itr)
    complex(kind(0d0)), intent(in) :: v(:)
    integer, intent(in) :: nsteps
    logical, intent(in) :: check_conv
    double precision, intent(out) :: alpha(:), beta(:), ene(8)
    integer, intent(out) :: itr
    integer(c_int) :: rc, done, cc
    cc = 0
    if (check_conv) cc = 1
    rc = pned_lanczos_run(g_ctx, v, int(nsteps, c_int), cc, alpha, beta, ene, done, 0_c_int)
    if (rc /= 0) stop 'pned_lanczos_run failed'
    itr = done
  end subroutine pned_lanczos_run_f

  !! parallelized_lncv1z: eigenvector x = sum_k coef(k) v_k from the stored alpha/beta of the first pass.
  subroutine pned_lncv1_f(v, nsteps, alpha, beta, coef, x)
    complex(kind(0d0)), intent(in) :: v(:)
    integer, intent(in) :: nsteps
    double precision, intent(in) :: alpha(:), beta(:), coef(:)
    complex(kind(0d0)), intent(out) :: x(:)
    if (pned_lanczos_vector(g_ctx, v, int(nsteps, c_int), alpha, beta, coef, x, 0_c_int) /= 0) &
        stop 'pned_lanczos_vector failed'
  end subroutine pned_lncv1_f

  !! parallelized_inv1 (inverse iteration with CG) for eigenvalue e from b.
  subroutine pned_inv1_f(e, b, x, inv_max, cg_max)
    double precision, intent(in) :: e
    complex(kind(0d0)), intent(in) :: b(:)
    complex(kind(0d0)), intent(out) :: x(:)
    integer, intent(in) :: inv_max, cg_max
    integer(c_int) :: ni, nc
    if (pned_cg_run(g_ctx, real(e, c_double), b, int(inv_max, c_int), int(cg_max, c_int), x, ni, nc, 0_c_int) /= 0) &
        stop 'pned_cg_run failed'
  end subroutine pned_inv1_f

  !! parallelized_TPSz for one seed on the model given to pned_gpu_init after
  !! change_to_TPS_hamiltonian (L = localHam_max); coef(nsteps, 5) as eval_phys_val.
  subroutine pned_tps_run_f(L, v, nsteps, alpha, beta, coef)
    double precision, intent(in) :: L
    complex(kind(0d0)), intent(in) :: v(:)
    integer, intent(in) :: nsteps
    double precision, intent(out) :: alpha(:), beta(:), coef(:, :)
    double precision, allocatable :: c_row(:)
    integer :: k, m
    allocate(c_row(5 * nsteps))
    if (pned_tps_run(g_ctx, real(L, c_double), v, int(nsteps, c_int), 0_c_int, c_null_ptr, alpha, beta, c_row, &
                     0_c_int) /= 0) stop 'pned_tps_run failed'
    do k = 1, nsteps
      do m = 1, 5
        coef(k, m) = c_row(5 * (k - 1) + m)
      end do
    end do
    deallocate(c_row)
  end subroutine pned_tps_run_f

  !! dump_alpha_beta_coef: SalphaSbeta file in the reference's layout.
  subroutine pned_dump_alpha_beta_coef_f(filename, alpha, beta, coef)
    character(len=*), intent(in) :: filename
    double precision, intent(in) :: alpha(:), beta(:), coef(:, :)
    if (pned_write_salphasbeta(trim(filename) // c_null_char, int(size(alpha), c_int), int(size(coef, 2), c_int), &
                               alpha, beta, coef) /= 0) stop 'pned_write_salphasbeta failed'
  end subroutine pned_dump_alpha_beta_coef_f

  !! The model of the same lattice and couplings in the sector of digit sum
  !! total_sz_target (for intalv_xy: total_sz + ipm), after pned_gpu_init.
  subroutine pned_gpu_init_target(n, q_spin, tree, ibond, parity_type, total_sz_target)
    integer, intent(in) :: n, q_spin, tree, ibond, parity_type, total_sz_target
    type(pned_model_desc) :: d
    integer(c_int) :: rc
    d%n_sites = n; d%q_spin = q_spin; d%tree = tree; d%n_bonds = ibond
    d%ipair = c_loc(g_ipair); d%bond_type = c_loc(g_btype)
    d%xlocal = c_loc(g_x); d%skip = c_loc(g_skip)
    d%parity_type = parity_type; d%total_sz = total_sz_target
    rc = pned_model_create(d, g_model2)
    if (rc /= 0) stop 'pned_model_create (target sector) failed'
    rc = pned_ctx_create(g_model2, 1_c_int, 0_c_size_t, g_ctx2)
    if (rc /= 0) stop 'pned_ctx_create (target sector) failed'
  end subroutine pned_gpu_init_target

  !! intalv_zz + parallelized_dsflnc1z for one momentum: qr(j) = q.r_j; salpha(1:nsteps),
  !! sbeta(1:nsteps+1) with sbeta(1) = cnorm, as the reference's DSF arrays.
  subroutine pned_dsf_zz_f(x, qr, nsteps, cnorm, salpha, sbeta)
    complex(kind(0d0)), intent(in) :: x(:)
    double precision, intent(in) :: qr(:)
    integer, intent(in) :: nsteps
    double precision, intent(out) :: cnorm, salpha(:), sbeta(:)
    double precision :: cn(1)
    if (pned_dsf_run(g_ctx, x, qr, int(nsteps, c_int), cn, salpha, sbeta, 0_c_int) /= 0) stop 'pned_dsf_run failed'
    cnorm = cn(1)
  end subroutine pned_dsf_zz_f

  !! intalv_xy ('xx'; Sa 'uu' ipm = 1, 'dd' ipm = -1) + parallelized_dsflnc1z: x on the
  !! pned_gpu_init model's basis, the chain on pned_gpu_init_target's.
  subroutine pned_dsf_xy_f(x, qr, nsteps, ipm, cnorm, salpha, sbeta)
    complex(kind(0d0)), intent(in) :: x(:)
    double precision, intent(in) :: qr(:)
    integer, intent(in) :: nsteps, ipm
    double precision, intent(out) :: cnorm, salpha(:), sbeta(:)
    double precision :: cn(1)
    if (pned_dsf_xy_run(g_ctx2, g_model, int(ipm, c_int), x, qr, int(nsteps, c_int), cn, salpha, sbeta, &
                        0_c_int) /= 0) stop 'pned_dsf_xy_run failed'
    cnorm = cn(1)
  end subroutine pned_dsf_xy_f

  !! The DSF driver's sq.txt line.
  subroutine pned_append_sq_f(filename, iq, q, norm)
    character(len=*), intent(in) :: filename
    integer, intent(in) :: iq
    double precision, intent(in) :: q(2), norm
    if (pned_append_sq(trim(filename) // c_null_char, int(iq, c_int), real(q(1), c_double), real(q(2), c_double), &
                       real(norm, c_double)) /= 0) stop 'pned_append_sq failed'
  end subroutine pned_append_sq_f

  !! dump_alpha_beta: SalphaSbeta_q... and vec_q... files in the reference's layout.
  subroutine pned_dump_alpha_beta_f(ab_file, vec_file, indx, sq, salpha, sbeta, v1, v2)
    character(len=*), intent(in) :: ab_file, vec_file
    integer, intent(in) :: indx
    complex(kind(0d0)), intent(in) :: sq
    double precision, intent(in) :: salpha(:), sbeta(:)
    complex(kind(0d0)), intent(in) :: v1(:), v2(:)
    if (pned_write_dsf_alpha_beta(trim(ab_file) // c_null_char, sq, salpha, sbeta, &
                                  int(size(salpha), c_int)) /= 0) stop 'pned_write_dsf_alpha_beta failed'
    if (pned_write_dsf_vectors(trim(vec_file) // c_null_char, int(indx, c_int), v1, v2, &
                               int(size(v1), c_int64_t)) /= 0) stop 'pned_write_dsf_vectors failed'
  end subroutine pned_dump_alpha_beta_f

  !! Lanczos run in steps that can stop and resume (interval_dump / interval_dump_read).
  subroutine pned_lanczos_begin_f(v, max_steps)
    complex(kind(0d0)), intent(in) :: v(:)
    integer, intent(in) :: max_steps
    if (pned_session_begin(g_ctx, 1_c_int, v, int(max_steps, c_int), 0d0, 0_c_int, c_null_ptr, 0_c_int) /= 0) &
        stop 'pned_session_begin failed'
  end subroutine pned_lanczos_begin_f

  subroutine pned_steps_f(nsteps)
    integer, intent(in) :: nsteps
    if (pned_session_step(g_ctx, int(nsteps, c_int)) /= 0) stop 'pned_session_step failed'
  end subroutine pned_steps_f

  subroutine pned_lanczos_read_f(alpha, beta, done)
    double precision, intent(out) :: alpha(:), beta(:)
    integer, intent(out) :: done
    integer(c_int) :: d, st
    if (pned_session_read(g_ctx, alpha, beta, c_null_ptr, d, st) /= 0) stop 'pned_session_read failed'
    done = d
  end subroutine pned_lanczos_read_f

  subroutine pned_interval_dump_f(filename)
    character(len=*), intent(in) :: filename
    if (pned_session_save(g_ctx, trim(filename) // c_null_char) /= 0) stop 'pned_session_save failed'
  end subroutine pned_interval_dump_f

  subroutine pned_interval_dump_read_f(filename, max_steps)
    character(len=*), intent(in) :: filename
    integer, intent(in) :: max_steps
    if (pned_session_load(g_ctx, trim(filename) // c_null_char, int(max_steps, c_int)) /= 0) &
        stop 'pned_session_load failed'
  end subroutine pned_interval_dump_read_f

  !! The GPU Lanczos run's state in parallelized_lnc1z's own variables at the top
  !! of its next iteration (v0 = H v_k - beta v_{k-1}, v1 = v_k), so that the
  !! reference's interval_dump writes its vecdump files unchanged (S1/2 Lanczos.f90:99-103).
  subroutine pned_lanczos_state_f(v0, v1)
    complex(kind(0d0)), intent(out) :: v0(:), v1(:)
    if (pned_session_lanczos_state(g_ctx, v0, v1, 0_c_int) /= 0) stop 'pned_session_lanczos_state failed'
  end subroutine pned_lanczos_state_f

  !! Resumes the GPU run from what interval_dump_read has read back (:87-93):
  !! alpha/beta of the done = itr_counter(1) - 1 steps, v0 and v1.
  subroutine pned_lanczos_resume_f(v0, v1, alpha, beta, done, max_steps)
    complex(kind(0d0)), intent(in) :: v0(:), v1(:)
    double precision, intent(in) :: alpha(:), beta(:)
    integer, intent(in) :: done, max_steps
    if (pned_session_begin_lanczos_at(g_ctx, v0, v1, alpha, beta, int(done, c_int), int(max_steps, c_int), &
                                      0_c_int) /= 0) stop 'pned_session_begin_lanczos_at failed'
  end subroutine pned_lanczos_resume_f

  subroutine pned_gpu_finalize()
    integer(c_int) :: rc
    if (c_associated(g_ctx2)) rc = pned_ctx_destroy(g_ctx2)
    if (c_associated(g_model2)) rc = pned_model_destroy(g_model2)
    if (c_associated(g_ctx)) rc = pned_ctx_destroy(g_ctx)
    if (c_associated(g_model)) rc = pned_model_destroy(g_model)
    g_ctx = c_null_ptr; g_model = c_null_ptr; g_ctx2 = c_null_ptr; g_model2 = c_null_ptr
  end subroutine pned_gpu_finalize
end module pned_gpu
