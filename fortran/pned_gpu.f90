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

  subroutine pned_gpu_finalize()
    integer(c_int) :: rc
    if (c_associated(g_ctx)) rc = pned_ctx_destroy(g_ctx)
    if (c_associated(g_model)) rc = pned_model_destroy(g_model)
    g_ctx = c_null_ptr; g_model = c_null_ptr
  end subroutine pned_gpu_finalize
end module pned_gpu
