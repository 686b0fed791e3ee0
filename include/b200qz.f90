! Fortran interface to libb200qz.so, the B200 multishift QZ that replaces
! the reference's PDHGEQZ on a 1x1 process grid.
!
! Two ways to call it from Fortran:
!  1. unchanged reference callers: CALL PDHGEQZ(...) resolves to the
!     exported symbol pdhgeqz_ when the program is linked against
!     libb200qz.so instead of libpdhgeqz.a (gfortran's default name
!     mangling: lower case plus one underscore, hidden CHARACTER lengths
!     appended by value);
!  2. callers that prefer explicit interfaces USE this module, which binds
!     the Fortran names to the C symbols with ISO_C_BINDING and does not
!     depend on any name-mangling convention.
module b200qz
  use iso_c_binding, only: c_int, c_double, c_char, c_size_t, c_ptr
  implicit none
  interface
     ! SUBROUTINE PDHGEQZ( JOB, COMPQ, COMPZ, N, ILO, IHI, H, DESCH, T, DESCT,
     !    ALPHAR, ALPHAI, BETA, Q, DESCQ, Z, DESCZ, DWORK, LDWORK, IWORK,
     !    LIWORK, INFO )  -- src/pdhgeqz/PDHGEQZ.f:15-31
     subroutine b200qz_pdhgeqz(job, compq, compz, n, ilo, ihi, h, desch, t, desct, &
          alphar, alphai, beta, q, descq, z, descz, dwork, ldwork, iwork, liwork, info, &
          len_job, len_compq, len_compz) bind(C, name="pdhgeqz_")
       import :: c_int, c_double, c_char, c_size_t
       character(kind=c_char), intent(in) :: job, compq, compz
       integer(c_int), intent(in) :: n, ilo, ihi
       real(c_double), intent(inout) :: h(*), t(*), q(*), z(*)
       integer(c_int), intent(in) :: desch(9), desct(9), descq(9), descz(9)
       real(c_double), intent(out) :: alphar(*), alphai(*), beta(*)
       real(c_double), intent(inout) :: dwork(*)
       integer(c_int), intent(in) :: ldwork, liwork
       integer(c_int), intent(inout) :: iwork(*)
       integer(c_int), intent(out) :: info
       integer(c_size_t), value :: len_job, len_compq, len_compz
     end subroutine b200qz_pdhgeqz

     ! SUBROUTINE KKQZCONF( EPS ) -- src/kkqz/kkqzconf.f:45-170 (accepted no-op)
     subroutine b200qz_kkqzconf(eps) bind(C, name="kkqzconf_")
       import :: c_double
       real(c_double), intent(in) :: eps
     end subroutine b200qz_kkqzconf

     ! context for the native entries below (one per device and host thread)
     integer(c_int) function b200qz_create(ctx, device) bind(C, name="b200qz_create")
       import :: c_int, c_ptr
       type(c_ptr), intent(out) :: ctx
       integer(c_int), value :: device
     end function b200qz_create
     subroutine b200qz_destroy(ctx) bind(C, name="b200qz_destroy")
       import :: c_ptr
       type(c_ptr), value :: ctx
     end subroutine b200qz_destroy

     ! balancing with DGGBAL's arguments (host arrays), the ILO/IHI producer
     ! the driver takes (PDHGEQZ.f:155-161); returns 0 or -i / 10001
     integer(c_int) function b200qz_ggbal_host(ctx, job, n, a, lda, b, ldb, ilo, ihi, lscale, rscale) &
          bind(C, name="b200qz_ggbal_host")
       import :: c_int, c_double, c_char, c_ptr
       type(c_ptr), value :: ctx
       character(kind=c_char), value :: job
       integer(c_int), value :: n, lda, ldb
       real(c_double), intent(inout) :: a(*), b(*)
       integer(c_int), intent(out) :: ilo, ihi
       real(c_double), intent(out) :: lscale(*), rscale(*)
     end function b200qz_ggbal_host

     ! back transformation with DGGBAK's arguments (host array v, n x m)
     integer(c_int) function b200qz_ggbak_host(ctx, job, side, n, ilo, ihi, lscale, rscale, m, v, ldv) &
          bind(C, name="b200qz_ggbak_host")
       import :: c_int, c_double, c_char, c_ptr
       type(c_ptr), value :: ctx
       character(kind=c_char), value :: job, side
       integer(c_int), value :: n, ilo, ihi, m, ldv
       real(c_double), intent(in) :: lscale(*), rscale(*)
       real(c_double), intent(inout) :: v(*)
     end function b200qz_ggbak_host

     ! reordering of the Schur form with DTGSEN's arguments (IJOB 0 or 1);
     ! the role of PDTGSEN (src/reorder/PDTGSEN.f:1)
     integer(c_int) function b200qz_gghrd_host(ctx, compq, compz, n, ilo, ihi, a, lda, b, ldb, q, ldq, z, ldz) &
          bind(C, name="b200qz_gghrd_host")
       import :: c_ptr, c_int, c_double, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char), value :: compq, compz
       integer(c_int), value :: n, ilo, ihi, lda, ldb, ldq, ldz
       real(c_double), intent(inout) :: a(lda, *), b(ldb, *), q(ldq, *), z(ldz, *)
     end function b200qz_gghrd_host
     integer(c_int) function b200qz_tgsen_host(ctx, ijob, wantq, wantz, select, n, s, lds, t, ldt, q, ldq, &
          z, ldz, alphar, alphai, beta, m, pl, pr, dif, info) bind(C, name="b200qz_tgsen_host")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: ijob, wantq, wantz, n, lds, ldt, ldq, ldz
       integer(c_int), intent(in) :: select(*)
       real(c_double), intent(inout) :: s(*), t(*), q(*), z(*)
       real(c_double), intent(out) :: alphar(*), alphai(*), beta(*)
       integer(c_int), intent(out) :: m, info
       real(c_double), intent(out) :: pl, pr
       real(c_double), intent(out) :: dif(2)
     end function b200qz_tgsen_host
  end interface
end module b200qz
