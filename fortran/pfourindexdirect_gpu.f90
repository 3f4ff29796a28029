! Drop-in replacement for SUBROUTINE FOURINDEX_ERI (src/pfourindexdirect.f90)
! of the polymer code: fills the C argument block of libpolymer_fock
! (include/polymer_fock.h, pfe_args) from the same modules the original reads
! and calls pfe_fourindex_eri.  Build: add pfourindexdirect_gpu.o in place of
! pfourindexdirect.o in the OBJS list of src/Makefile and link with
! -lpolymer_fock -lcudart.
MODULE PFE_BINDING
   USE ISO_C_BINDING
   IMPLICIT NONE
   TYPE, BIND(C) :: PFE_ARGS
      INTEGER(C_INT32_T) :: NPGS, NCGS, NPSHELL, LMAX
      TYPE(C_PTR) :: P_SHELL, P_SHELL_ANG, PGSX, PGSY, PGSZ, ZT, CC, C2H
      TYPE(C_PTR) :: S_P, P_P, P_P_HELIX, IGAMMA
      INTEGER(C_INT32_T) :: CEL1(3), CEL2(3), REDUCED_CEL1(3)
      REAL(C_DOUBLE) :: PERIOD(3), HELIX, INTTOL
      INTEGER(C_INT32_T) :: PRINT_LEVEL, MYID, NUMPROCS, PRECISION_MODE
      REAL(C_DOUBLE) :: MIXED_CUTOFF
   END TYPE
   INTERFACE
      INTEGER(C_INT32_T) FUNCTION PFE_FOURINDEX_ERI(A, C_C, X_C) BIND(C, NAME='pfe_fourindex_eri')
         IMPORT :: PFE_ARGS, C_INT32_T, C_DOUBLE
         TYPE(PFE_ARGS), INTENT(IN) :: A
         REAL(C_DOUBLE) :: C_C(*), X_C(*)
      END FUNCTION
      INTEGER(C_INT32_T) FUNCTION PFE_LAST_ERROR(BUF, N) BIND(C, NAME='pfe_last_error')
         IMPORT :: C_CHAR, C_INT32_T
         CHARACTER(KIND=C_CHAR) :: BUF(*)
         INTEGER(C_INT32_T), VALUE :: N
      END FUNCTION
   END INTERFACE
CONTAINS
   ! C_LOC needs an argument with TARGET (or POINTER); the module arrays are
   ! plain ALLOCATABLE, so their addresses are taken through a TARGET dummy.
   ! A contiguous actual array is passed by its address, and the library reads
   ! it only during the call below, while the array is still allocated.
   FUNCTION DADDR(X) RESULT(P)
      REAL(C_DOUBLE), TARGET, INTENT(IN) :: X(*)
      TYPE(C_PTR) :: P
      P = C_LOC(X(1))
   END FUNCTION
END MODULE

SUBROUTINE FOURINDEX_ERI
   USE MPI_F08
   USE ISO_C_BINDING
   USE PFE_BINDING
   USE CONSTANTS
   USE CONTROL
   USE STRUCTURE
   USE BASISSET
   USE INTEGRAL
   USE FMT
   IMPLICIT NONE
   TYPE(PFE_ARGS) :: A
   INTEGER(C_INT32_T) :: RC
   INTEGER, ALLOCATABLE, TARGET :: PS(:,:,:,:), PA(:)
   CHARACTER(KIND=C_CHAR) :: MSG(512)
   CHARACTER(LEN=512) :: TXT
   INTEGER :: I, N

   ALLOCATE(PS, SOURCE=P_SHELL)            ! default INTEGER is C_INT32_T with gfortran
   ALLOCATE(PA, SOURCE=P_SHELL_ANG)
   A%NPGS = NPGS; A%NCGS = NCGS; A%NPSHELL = NPSHELL; A%LMAX = BASIS_LMAX
   A%P_SHELL = C_LOC(PS); A%P_SHELL_ANG = C_LOC(PA)
   A%PGSX = DADDR(PGSX); A%PGSY = DADDR(PGSY); A%PGSZ = DADDR(PGSZ); A%ZT = DADDR(ZT)
   A%CC = DADDR(CC); A%C2H = DADDR(C2H); A%S_P = DADDR(S_P); A%P_P = DADDR(P_P)
   A%P_P_HELIX = DADDR(P_P_HELIX); A%IGAMMA = DADDR(IGAMMA)
   A%CEL1 = (/CEL1X, CEL1Y, CEL1Z/); A%CEL2 = (/CEL2X, CEL2Y, CEL2Z/)
   A%REDUCED_CEL1 = (/REDUCED_CEL1X, REDUCED_CEL1Y, REDUCED_CEL1Z/)
   A%PERIOD = (/PERIODX, PERIODY, PERIODZ/); A%HELIX = HELIX; A%INTTOL = DOPTN(12)
   A%PRINT_LEVEL = IOPTN(9); A%MYID = MYID; A%NUMPROCS = NUMPROCS
   A%PRECISION_MODE = 0; A%MIXED_CUTOFF = 0.0D0

   RC = PFE_FOURINDEX_ERI(A, C_C, X_C)     ! this rank's share of C_C, X_C
   IF (RC /= 0) THEN
      N = PFE_LAST_ERROR(MSG, 512)
      TXT = ''
      DO I = 1, MIN(N, 512)
         TXT(I:I) = MSG(I)
      ENDDO
      CALL PABORT('GPU FOURINDEX_ERI FAILED: '//TRIM(TXT))
   ENDIF
   ! the reference all-reduces primitive J/K (src/pfourindexdirect.f90:757-758);
   ! the contraction is linear, so summing the contracted shares is the same
   CALL MPI_ALLREDUCE(MPI_IN_PLACE, C_C, SIZE(C_C), MPI_DOUBLE_PRECISION, MPI_SUM, MPI_COMM_WORLD, IERR)
   CALL MPI_ALLREDUCE(MPI_IN_PLACE, X_C, SIZE(X_C), MPI_DOUBLE_PRECISION, MPI_SUM, MPI_COMM_WORLD, IERR)
   IF (IOPTN(9) >= 2) THEN
      WRITE(6,'(A)') 'COULOMB MATRIX FOR CONTRACTED GAUSSIANS'
      CALL DUMP1(C_C, NCGS, CEL1X, CEL1Y, CEL1Z)
      WRITE(6,'(A)') 'EXCHANGE MATRIX FOR CONTRACTED GAUSSIANS'
      CALL DUMP1(X_C, NCGS, CEL1X, CEL1Y, CEL1Z)
   ENDIF
   DEALLOCATE(PS, PA)
END SUBROUTINE
