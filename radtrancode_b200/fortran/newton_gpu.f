C----------------------------------------------------------------------
C     The optimal-estimation step of nemesis/coreret.f on the B200, as
C     drop-in replacements with the reference's names and arguments:
C       calc_phiret       nemesis/calc_phiret.f:1 (coreret.f:557, 960)
C       calc_gain_matrix  nemesis/calc_gain_matrix.f:1
C                         (coreret.f:554, 997)
C       calcnextxn        nemesis/calcnextxn.f:1 (coreret.f:609)
C     Each runs on the device in FP64 through the C ABI of
C     include/radtran_b200.h.  The library takes the diagonal of Se^-1
C     (NEMESIS builds Se from the per-point errors of the .spx file, so
C     it is diagonal); a non-zero off-diagonal element stops the run
C     with a message rather than being dropped.
C
C     Not built here (no Fortran compiler on this build host).  Compile
C     from nemesis/ after radtran_b200.f90 (the INCLUDE paths are the
C     reference's) and link the object before the nemesis archive.
C----------------------------------------------------------------------
      REAL FUNCTION calc_phiret(ny, y, yn, sei, nx, xn, xa, sai, chisq)
      USE radtran_b200
      IMPLICIT NONE
      INCLUDE '../radtran/includes/arrdef.f'
      INCLUDE 'arraylen.f'
      INTEGER nx, ny, i, j
      REAL y(my), yn(my), xn(mx), xa(mx), chisq
      DOUBLE PRECISION sei(my,my), sai(mx,mx)
      DOUBLE PRECISION, ALLOCATABLE :: sed(:), sac(:)
      REAL(c_float) phi(1), chi(1)
      INTEGER(c_int) st
      CALL rtb_context_open()
      ALLOCATE(sed(ny), sac(nx*nx))
      CALL se_diagonal(ny, sei, sed, 'CALC_PHIRET')
C     Sa^-1 without its leading dimension (symmetric: either order)
      DO j = 1, nx
        DO i = 1, nx
          sac(i + nx*(j - 1)) = sai(i,j)
        ENDDO
      ENDDO
      st = rtb_calc_phiret_batch(ctx, 1, nx, ny, y, yn, sed, xn, xa,
     1  sac, phi, chi)
      CALL rtb_check(st, 'CALC_PHIRET')
      chisq = chi(1)
      calc_phiret = phi(1)
      DEALLOCATE(sed, sac)
      RETURN
      END

      SUBROUTINE calc_gain_matrix(nx, ny, kk_in, sx_in, sxi, se_in,
     1  sei, dd_out, aa_out)
      USE radtran_b200
      IMPLICIT NONE
      INCLUDE '../radtran/includes/arrdef.f'
      INCLUDE 'arraylen.f'
      INTEGER nx, ny
      REAL kk_in(my,mx), sx_in(mx,mx), se_in(my,my)
      DOUBLE PRECISION sxi(mx,mx), sei(my,my)
      DOUBLE PRECISION dd_out(mx,my), aa_out(mx,mx)
      DOUBLE PRECISION, ALLOCATABLE :: sed(:)
      INTEGER(c_int) st, nonpd
      CALL rtb_context_open()
      ALLOCATE(sed(ny))
      CALL se_diagonal(ny, sei, sed, 'CALC_GAIN_MATRIX')
      st = rtb_calc_gain_matrix(ctx, nx, ny, mx, my, kk_in, sxi, sed,
     1  dd_out, aa_out, nonpd)
      CALL rtb_check(st, 'CALC_GAIN_MATRIX')
      DEALLOCATE(sed)
      RETURN
      END

      SUBROUTINE calcnextxn(nx, ny, x0_in, xn_in, y_in, yn_in, dd_in,
     1  aa_in, x_out)
      USE radtran_b200
      IMPLICIT NONE
      INCLUDE '../radtran/includes/arrdef.f'
      INCLUDE 'arraylen.f'
      INTEGER nx, ny
      REAL x0_in(mx), xn_in(mx), y_in(my), yn_in(my), x_out(mx)
      DOUBLE PRECISION dd_in(mx,my), aa_in(mx,mx)
      INTEGER(c_int) st
      CALL rtb_context_open()
      st = rtb_calcnextxn(ctx, nx, ny, mx, x0_in, xn_in, y_in, yn_in,
     1  dd_in, aa_in, x_out)
      CALL rtb_check(st, 'CALCNEXTXN')
      RETURN
      END

C     the diagonal of sei(1:ny,1:ny); an off-diagonal element stops
      SUBROUTINE se_diagonal(ny, sei, sed, who)
      IMPLICIT NONE
      INCLUDE '../radtran/includes/arrdef.f'
      INCLUDE 'arraylen.f'
      INTEGER ny, i, j
      DOUBLE PRECISION sei(my,my), sed(ny)
      CHARACTER*(*) who
      DO j = 1, ny
        DO i = 1, ny
          IF (i .NE. j .AND. sei(i,j) .NE. 0.0D0) THEN
            PRINT*, who, ' (B200): Se^-1 is not diagonal at ', i, j
            STOP
          ENDIF
        ENDDO
        sed(j) = sei(j,j)
      ENDDO
      RETURN
      END
