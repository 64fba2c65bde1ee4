! kaos_gpu_iface.f90 -- ISO_C_BINDING interface of libkaos_gpu (the C-ABI in
! include/kaos_gpu.h) for a Fortran host that keeps KAOS's _ModelInput /
! _KineticMainParams parameterisation and replaces the body of
! KineticSolverSub (_8_KineticSolver.f90:54-239) by calls into the B200
! library.  The derived types mirror the C structs field by field
! (bind(C) layout); flag names follow _ModelInput.f90.
!
! Build (where a Fortran compiler exists):
!   gfortran -c kaos_gpu_iface.f90
!   gfortran host.f90 kaos_gpu_iface.o -L<repo>/kaos_b200 -lkaos_gpu -lcudart
module kaos_gpu_iface
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: KAOS_OK = 0, KAOS_ERR_PARAM = 1, &
    KAOS_ERR_CAPACITY = 2, KAOS_ERR_NAN = 3, KAOS_ERR_CUDA = 4, &
    KAOS_ERR_TIMEOUT = 5, KAOS_ERR_STATE = 6
  integer(c_int), parameter :: KAOS_PREC_FP64 = 0, KAOS_PREC_MIXED = 1, &
                                KAOS_PREC_MIXED_K64 = 2
  integer(c_int), parameter :: KAOS_M0 = 0, KAOS_M1PERP1 = 1, &
    KAOS_M1PERP2 = 2, KAOS_M1PAR = 3, KAOS_M2 = 4, KAOS_M2PERP1 = 5, &
    KAOS_M2PERP2 = 6, KAOS_M2PAR = 7, KAOS_M1PERP = 8, KAOS_M2PERP = 9, &
    KAOS_NQ = 10, KAOS_EAMAG = 11, KAOS_EGMAG = 12, KAOS_M0FILT = 13, &
    KAOS_NUPOI = 14, KAOS_ENA_NQ = 15, KAOS_ENA_M0 = 16, KAOS_ENA_M1P = 17, &
    KAOS_ENA_M1Q = 18, KAOS_ENA_M1PHI = 19, KAOS_ENA_M2 = 20, &
    KAOS_ENA_M2P = 21, KAOS_ENA_M2Q = 22, KAOS_ENA_M2PHI = 23

  ! kaos_params_c
  type, bind(C) :: kaos_params_t
    real(c_double) :: ms, qs, h, mNeut, TNeut, dNTe, dNTeEND
    integer(c_int64_t) :: seed
    integer(c_int32_t) :: ndatfac, precision, ION2VPERPflag, ICRflag, &
      ICRCOHERENCEflag, MIRRORflag, GRAVflag, EAMBflag, EAMBSIGNflag, &
      EAMBSELFCONSISTflag, EAPRESSUREflag, MOMENTFILTERflag, QEXCHANGEflag, &
      LBCONDITIONflag, UBCONDITIONflag, STATICINJECTIONflag, &
      PHASEENERGYPARIONMOMENTCENTERflag, PHASEENERGYPERPIONMOMENTCENTERflag, &
      M0MAfilterPt, M1ParMAfilterPt, M1Perp1MAfilterPt, M1Perp2MAfilterPt, &
      M2ParMAfilterPt
    integer(c_int32_t) :: FLUXINJECTIONflag
    integer(c_int32_t) :: reserved(3)
  end type kaos_params_t

  ! kaos_tube_c: pointers are c_loc() of the FluxTubeT per-cell tables
  ! (cells NqLB..NqUB, contiguous, first index = NqLB)
  type, bind(C) :: kaos_tube_t
    integer(c_int32_t) :: nq, capacity
    real(c_double) :: pG, phiG, nsnormfac, nsnormCLB, nsnormCUB, sumdsICR
    type(c_ptr) :: qGL, qGH, qGC, hqC, dqC, d3xC, rGC, thetaGC, ellGC
    type(c_ptr) :: TeG, TsG, nsnormCNeut
    type(c_ptr) :: lambdaPerp, EtaLH, XiPerp1, XiPerp2
    type(c_ptr) :: S0, OmegaG0, ChiPerp1, ChiPerp2
    real(c_double) :: ms, qs   ! SpecieT(s)%msT, qsT of this entry; 0 = params
  end type kaos_tube_t

  ! kaos_vgrid_c: separable velocity-cell edges (n+1 values per axis)
  type, bind(C) :: kaos_vgrid_t
    integer(c_int32_t) :: n1, n2, npar
    type(c_ptr) :: e1, e2, epar
  end type kaos_vgrid_t

  ! kaos_init_c: on-device initial ions
  type, bind(C) :: kaos_init_t
    type(c_ptr) :: counts            ! integer(c_int64_t) per cell
    real(c_double) :: tail_fraction, kappa, tail_T
    integer(c_int64_t) :: seed
  end type kaos_init_t

  interface
    integer(c_int) function kaos_create(p, tubes, ntubes, vg, h) &
        bind(C, name="kaos_create")
      import :: c_int, c_int32_t, c_ptr, kaos_params_t, kaos_tube_t, kaos_vgrid_t
      type(kaos_params_t), intent(in) :: p
      type(kaos_tube_t), intent(in) :: tubes(*)
      integer(c_int32_t), value :: ntubes
      type(kaos_vgrid_t), intent(in) :: vg
      type(c_ptr), intent(out) :: h
    end function kaos_create

    integer(c_int) function kaos_load_particles(h, tube, q, vpar, vperp1, &
        vperp2, n) bind(C, name="kaos_load_particles")
      import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      real(c_double), intent(in) :: q(*), vpar(*), vperp1(*), vperp2(*)
      integer(c_int64_t), value :: n
    end function kaos_load_particles

    integer(c_int) function kaos_init_particles(h, tube, init) &
        bind(C, name="kaos_init_particles")
      import :: c_int, c_int32_t, c_ptr, kaos_init_t
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      type(kaos_init_t), intent(in) :: init
    end function kaos_init_particles

    integer(c_int) function kaos_set_fields(h, tube, EAmag, nq) &
        bind(C, name="kaos_set_fields")
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube, nq
      real(c_double), intent(in) :: EAmag(*)
    end function kaos_set_fields

    integer(c_int) function kaos_step(h, nsteps) bind(C, name="kaos_step")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), value :: nsteps
    end function kaos_step

    integer(c_int) function kaos_get_step(h, n) bind(C, name="kaos_get_step")
      import :: c_int, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int64_t), intent(out) :: n
    end function kaos_get_step

    integer(c_int) function kaos_get_count(h, tube, nion, nena) &
        bind(C, name="kaos_get_count")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      integer(c_int64_t), intent(out) :: nion, nena
    end function kaos_get_count

    integer(c_int) function kaos_get_moments(h, tube, which, out, nq) &
        bind(C, name="kaos_get_moments")
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube, which, nq
      real(c_double), intent(out) :: out(*)
    end function kaos_get_moments

    integer(c_int) function kaos_get_moments_all(h, tube, out, nq) &
        bind(C, name="kaos_get_moments_all")
      import :: c_int, c_int32_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube, nq
      real(c_double), intent(out) :: out(*)
    end function kaos_get_moments_all

    integer(c_int) function kaos_get_counts(h, tube, out, nbins) &
        bind(C, name="kaos_get_counts")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      integer(c_int64_t), intent(out) :: out(*)
      integer(c_int64_t), value :: nbins
    end function kaos_get_counts

    integer(c_int) function kaos_set_export(h, on) bind(C, name="kaos_set_export")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: on
    end function kaos_set_export

    integer(c_int) function kaos_get_particles(h, tube, q, vpar, vperp1, &
        vperp2, qind, n) bind(C, name="kaos_get_particles")
      import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      real(c_double), intent(out) :: q(*), vpar(*), vperp1(*), vperp2(*)
      integer(c_int32_t), intent(out) :: qind(*)
      integer(c_int64_t), value :: n
    end function kaos_get_particles

    integer(c_int) function kaos_get_positions(h, tube, rho, z, n) &
        bind(C, name="kaos_get_positions")
      import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      real(c_double), intent(out) :: rho(*), z(*)
      integer(c_int64_t), value :: n
    end function kaos_get_positions

    integer(c_int) function kaos_get_enas(h, tube, x, y, z, vx, vy, vz, n) &
        bind(C, name="kaos_get_enas")
      import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      real(c_double), intent(out) :: x(*), y(*), z(*), vx(*), vy(*), vz(*)
      integer(c_int64_t), value :: n
    end function kaos_get_enas

    integer(c_int) function kaos_get_boundary(h, tube, lb_out, ub_out, &
        lb_in, ub_in) bind(C, name="kaos_get_boundary")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      integer(c_int64_t), intent(out) :: lb_out, ub_out, lb_in, ub_in
    end function kaos_get_boundary

    integer(c_int) function kaos_get_boundary_ena(h, tube, lb_out, ub_out) &
        bind(C, name="kaos_get_boundary_ena")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      integer(c_int64_t), intent(out) :: lb_out, ub_out
    end function kaos_get_boundary_ena

    integer(c_int) function kaos_get_timing(h, ms, launches) &
        bind(C, name="kaos_get_timing")
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      real(c_double), intent(out) :: ms
      integer(c_int64_t), intent(out) :: launches
    end function kaos_get_timing

    integer(c_int) function kaos_get_push_timing(h, ms, launches) &
        bind(C, name="kaos_get_push_timing")
      import :: c_int, c_int64_t, c_double, c_ptr
      type(c_ptr), value :: h
      real(c_double), intent(out) :: ms
      integer(c_int64_t), intent(out) :: launches
    end function kaos_get_push_timing

    integer(c_int) function kaos_set_graph(h, on) bind(C, name="kaos_set_graph")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: on
    end function kaos_set_graph

    integer(c_int) function kaos_set_launch(h, chunk, mode) &
        bind(C, name="kaos_set_launch")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: chunk, mode
    end function kaos_set_launch

    integer(c_int) function kaos_set_ena_grid(h, vg) bind(C, name="kaos_set_ena_grid")
      import :: c_int, c_ptr, kaos_vgrid_t
      type(c_ptr), value :: h
      type(kaos_vgrid_t), intent(in) :: vg
    end function kaos_set_ena_grid

    integer(c_int) function kaos_set_reduce(h, fn, ctx) bind(C, name="kaos_set_reduce")
      import :: c_int, c_ptr, c_funptr
      type(c_ptr), value :: h
      type(c_funptr), value :: fn
      type(c_ptr), value :: ctx
    end function kaos_set_reduce

    integer(c_int) function kaos_update_tube(h, tube, t) bind(C, name="kaos_update_tube")
      import :: c_int, c_int32_t, c_ptr, kaos_tube_t
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      type(kaos_tube_t), intent(in) :: t
    end function kaos_update_tube

    integer(c_int) function kaos_set_rank(h, rank, nranks) bind(C, name="kaos_set_rank")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: rank, nranks
    end function kaos_set_rank

    integer(c_int) function kaos_set_id_base(h, tube, base) bind(C, name="kaos_set_id_base")
      import :: c_int, c_int32_t, c_int64_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), value :: tube
      integer(c_int64_t), value :: base
    end function kaos_set_id_base

    integer(c_int) function kaos_get_launch(h, chunk, mode) &
        bind(C, name="kaos_get_launch")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), intent(out) :: chunk, mode
    end function kaos_get_launch

    type(c_ptr) function kaos_last_error(h) bind(C, name="kaos_last_error")
      import :: c_ptr
      type(c_ptr), value :: h
    end function kaos_last_error

    integer(c_int) function kaos_get_status(h, status) bind(C, name="kaos_get_status")
      import :: c_int, c_int32_t, c_ptr
      type(c_ptr), value :: h
      integer(c_int32_t), intent(out) :: status
    end function kaos_get_status

    subroutine kaos_destroy(h) bind(C, name="kaos_destroy")
      import :: c_ptr
      type(c_ptr), value :: h
    end subroutine kaos_destroy

    ! statistics without device allocation: every array but p and vg is a
    ! device pointer (c_ptr from the host's own device allocator);
    ! d_moments holds [11][nq] doubles, d_counts nq int64 or c_null_ptr
    integer(c_int) function kaos_moments_noalloc(p, vg, nq, d_qedges, d_d3x, &
        nsnormfac, d_q, d_vpar, d_vperp1, d_vperp2, n, d_moments, d_counts, &
        stream) bind(C, name="kaos_moments_noalloc")
      import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr, kaos_params_t, &
                kaos_vgrid_t
      type(kaos_params_t), intent(in) :: p
      type(kaos_vgrid_t), intent(in) :: vg
      integer(c_int32_t), value :: nq
      type(c_ptr), value :: d_qedges, d_d3x
      real(c_double), value :: nsnormfac
      type(c_ptr), value :: d_q, d_vpar, d_vperp1, d_vperp2
      integer(c_int64_t), value :: n
      type(c_ptr), value :: d_moments, d_counts, stream
    end function kaos_moments_noalloc

    ! diagnostic sampler of the device generators; out: host array of
    ! 4 (Philox words), 2 (Gaussian pairs) or 1 (Poisson) doubles per draw
    integer(c_int) function kaos_sample_rng(kind, seed, id0, step, c3, lambda, &
        n, out) bind(C, name="kaos_sample_rng")
      import :: c_int, c_int32_t, c_int64_t, c_double
      integer(c_int32_t), value :: kind
      integer(c_int64_t), value :: seed, id0
      integer(c_int32_t), value :: step, c3
      real(c_double), value :: lambda
      integer(c_int64_t), value :: n
      real(c_double), intent(out) :: out(*)
    end function kaos_sample_rng

    type(c_ptr) function kaos_version() bind(C, name="kaos_version")
      import :: c_ptr
    end function kaos_version
  end interface

end module kaos_gpu_iface
