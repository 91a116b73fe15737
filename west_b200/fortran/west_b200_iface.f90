!
! Fortran binding of libwestb200.so for WEST's wstat.x (iso_c_binding).
!
! Replaces the CALL dfpt(...) of Wstat/apply_operator.f90:58 by
! CALL west_b200_apply_operator(...) when WEST is built with -D__WEST_B200.
! Compiles inside a WEST/QE tree (it USEs QE and WEST modules); it is not
! compiled by this repository, which has no Fortran compiler.
!
MODULE west_b200_iface
  !
  USE iso_c_binding
  !
  IMPLICIT NONE
  !
  TYPE, BIND(C) :: wb_system
     INTEGER(C_INT) :: npw, npwx, nr1, nr2, nr3
     INTEGER(C_INT) :: nbnd_occ, nkb, n_dfpt_maxiter, l_kinetic_only, gstart
     TYPE(C_PTR) :: nl, nlm, g2kin, vrs, evc, et, occupation, vkb, deeq, sqvc
     REAL(C_DOUBLE) :: alpha_pv, omega, wk
  END TYPE
  !
  INTERFACE
     INTEGER(C_INT) FUNCTION wb_ctx_create(ctx, sys, device) BIND(C, NAME='wb_ctx_create')
       IMPORT :: C_INT, C_PTR, wb_system
       TYPE(C_PTR), INTENT(OUT) :: ctx
       TYPE(wb_system), INTENT(IN) :: sys
       INTEGER(C_INT), VALUE :: device
     END FUNCTION
     INTEGER(C_INT) FUNCTION wb_ctx_destroy(ctx) BIND(C, NAME='wb_ctx_destroy')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
     END FUNCTION
     INTEGER(C_INT) FUNCTION wb_apply_operator(ctx, m, dvg, ld_dvg, dng, ld_dng, tr2, iq, unconverged) &
          & BIND(C, NAME='wb_apply_operator')
       IMPORT :: C_INT, C_PTR, C_DOUBLE, C_DOUBLE_COMPLEX
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: m, ld_dvg, ld_dng, iq
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(IN) :: dvg(*)
       COMPLEX(C_DOUBLE_COMPLEX), INTENT(OUT) :: dng(*)
       REAL(C_DOUBLE), VALUE :: tr2
       INTEGER(C_INT), INTENT(OUT) :: unconverged(*)
     END FUNCTION
     INTEGER(C_INT) FUNCTION wb_set_precision(ctx, mode) BIND(C, NAME='wb_set_precision')
       IMPORT :: C_INT, C_PTR
       TYPE(C_PTR), VALUE :: ctx
       INTEGER(C_INT), VALUE :: mode
     END FUNCTION
     FUNCTION wb_last_error() BIND(C, NAME='wb_last_error')
       IMPORT :: C_PTR
       TYPE(C_PTR) :: wb_last_error
     END FUNCTION
  END INTERFACE
  !
  TYPE(C_PTR), SAVE :: wb_ctx = C_NULL_PTR
  ! host copies that must outlive wb_ctx_create (it copies them to the device)
  INTEGER(C_INT), ALLOCATABLE, TARGET, SAVE :: nl_c(:), nlm_c(:)
  REAL(C_DOUBLE), ALLOCATABLE, TARGET, SAVE :: g2kin_c(:), vrs_c(:), et_c(:), occ_c(:), deeq_c(:,:), sqvc_c(:)
  COMPLEX(C_DOUBLE_COMPLEX), ALLOCATABLE, TARGET, SAVE :: evc_c(:,:), vkb_c(:,:)
  !
CONTAINS
  !
  !-----------------------------------------------------------------------
  SUBROUTINE west_b200_init()
    !-----------------------------------------------------------------------
    ! Gathers what dfpt reads (dfpt_module.f90:93-225) for k-point 1, Gamma.
    !
    USE kinds,              ONLY : DP
    USE fft_base,           ONLY : dffts
    USE gvect,              ONLY : gstart
    USE pwcom,              ONLY : npw, npwx, ngk
    USE wvfct,              ONLY : g2kin, et
    USE scf,                ONLY : vrs
    USE wavefunctions,      ONLY : evc
    USE uspp,               ONLY : nkb, vkb, deeq, indv_ijkb0
    USE uspp_param,         ONLY : nh
    USE ions_base,          ONLY : nat, ityp
    USE uspp_init,          ONLY : init_us_2
    USE cell_base,          ONLY : omega
    USE klist,              ONLY : igk_k
    USE westcom,            ONLY : nbnd_occ, occupation, alphapv_dfpt, n_dfpt_maxiter, l_kinetic_only
    USE types_bz_grid,      ONLY : k_grid
    USE types_coulomb,      ONLY : pot3D
    !
    TYPE(wb_system), TARGET :: s
    INTEGER :: na, ih, jh, ikb, jkb, nb
    INTEGER(C_INT) :: ierr
    !
    nb = nbnd_occ(1)
    npw = ngk(1)                               ! as dfpt_module.f90:34,175 (pwcom's npw)
    CALL g2_kin(1)                             ! dfpt_module.f90:153
    IF (nkb > 0) CALL init_us_2(npw, igk_k(1,1), k_grid%p_cart(1,1), vkb, .FALSE.)   ! :158-160, host vkb
    ALLOCATE(nl_c(npw), nlm_c(npw), g2kin_c(npw), vrs_c(dffts%nnr), et_c(nb), occ_c(nb))
    ALLOCATE(deeq_c(MAX(nkb,1), MAX(nkb,1)), sqvc_c(npw), evc_c(npwx, nb), vkb_c(npwx, MAX(nkb,1)))
    nl_c = dffts%nl(1:npw); nlm_c = dffts%nlm(1:npw)
    g2kin_c = g2kin(1:npw); vrs_c = vrs(:,1); et_c = et(1:nb,1); occ_c = occupation(1:nb,1)
    sqvc_c = pot3D%sqvc(1:npw)
    evc_c = evc(:,1:nb)
    deeq_c = 0._DP
    IF (nkb > 0) THEN
       vkb_c = vkb(:,1:nkb)
       DO na = 1, nat                         ! dense nkb x nkb from QE's per-atom blocks
          DO ih = 1, nh(ityp(na))
             DO jh = 1, nh(ityp(na))
                ikb = indv_ijkb0(na) + ih
                jkb = indv_ijkb0(na) + jh
                deeq_c(ikb, jkb) = deeq(ih, jh, na, 1)
             ENDDO
          ENDDO
       ENDDO
    ENDIF
    s%npw = npw; s%npwx = npwx
    s%nr1 = dffts%nr1; s%nr2 = dffts%nr2; s%nr3 = dffts%nr3
    s%nbnd_occ = nb; s%nkb = nkb; s%n_dfpt_maxiter = n_dfpt_maxiter
    s%l_kinetic_only = MERGE(1, 0, l_kinetic_only); s%gstart = gstart
    s%nl = C_LOC(nl_c); s%nlm = C_LOC(nlm_c); s%g2kin = C_LOC(g2kin_c); s%vrs = C_LOC(vrs_c)
    s%evc = C_LOC(evc_c); s%et = C_LOC(et_c); s%occupation = C_LOC(occ_c)
    s%vkb = C_LOC(vkb_c); s%deeq = C_LOC(deeq_c); s%sqvc = C_LOC(sqvc_c)
    s%alpha_pv = REAL(alphapv_dfpt, KIND=DP); s%omega = omega; s%wk = k_grid%weight(1)
    ierr = wb_ctx_create(wb_ctx, s, 0_C_INT)
    IF (ierr /= 0) CALL errore('west_b200_init', 'wb_ctx_create failed', INT(-ierr))
    !
  END SUBROUTINE
  !
  !-----------------------------------------------------------------------
  SUBROUTINE west_b200_apply_operator(m, dvg, dng, tr2, iq)
    !-----------------------------------------------------------------------
    ! Drop-in for apply_operator (Wstat/apply_operator.f90:14).
    !
    USE kinds,     ONLY : DP
    USE io_global, ONLY : stdout
    USE westcom,   ONLY : npwqx
    !
    INTEGER, INTENT(IN) :: m, iq
    COMPLEX(DP), INTENT(IN) :: dvg(npwqx, m)
    COMPLEX(DP), INTENT(OUT) :: dng(npwqx, m)
    REAL(DP), INTENT(IN) :: tr2
    INTEGER(C_INT) :: ierr
    INTEGER(C_INT), ALLOCATABLE :: unconv(:)
    INTEGER :: ipert
    !
    IF (.NOT. C_ASSOCIATED(wb_ctx)) CALL west_b200_init()
    ALLOCATE(unconv(MAX(m,1)))
    ierr = wb_apply_operator(wb_ctx, INT(m, C_INT), dvg, INT(npwqx, C_INT), dng, INT(npwqx, C_INT), &
         & REAL(tr2, C_DOUBLE), INT(iq, C_INT), unconv)
    IF (ierr /= 0) CALL errore('west_b200_apply_operator', 'wb_apply_operator failed', INT(-ierr))
    DO ipert = 1, m                            ! dfpt_module.f90:358-359
       IF (unconv(ipert) /= 0) WRITE(stdout, '(7X,"** WARNING : PERT ",I8," iks ",I8," not converged, ierr = ",I8)') &
          & ipert, 1, unconv(ipert)
    ENDDO
    DEALLOCATE(unconv)
    !
  END SUBROUTINE
  !
END MODULE
