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
  end interface
end module b200qz
