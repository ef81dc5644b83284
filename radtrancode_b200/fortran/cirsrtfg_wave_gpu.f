C----------------------------------------------------------------------
C     CIRSRTFG_WAVE on the B200: drop-in replacement of
C     radtran/cirsradg/cirsrtfg_wave.f (same name and arguments,
C     cirsrtfg_wave.f:1-3).
C
C     The reference's set-up stays as it is: the .fwh and .lte files,
C     SUBPATHG (layers, paths, the /LGRAD/ gradient matrices).  In place
C     of READ_KLIST and the wavenumber loop over CIRSRADG_WAVE
C     (cirsrtfg_wave.f:222-516) the /PATHVA/, /LAYCOM/ and /LGRAD/
C     arrays go to rtb_cirsrtfg_wave with their MAXLAY / MAXCON / MAXV
C     leading dimensions; the library computes every wavenumber and the
C     convolution onto the channels and packs the outputs as
C     cirsrtfg_wave.f:425-446, 448-516 do.
C
C     Tables, loaded once per run and kept on the device: the .kta files
C     of <runname>.kls in their listed order (every gas takes the
C     library's per-wavenumber choice among its tables, RTB_KTAB_BY_ID,
C     as READ_KLIST assigns lun(iwave, igas)), the CIA table of
C     /CIATABLE/ (ANAME1, DNU1), and with FLAGH2P = 1 the para-H2 table
C     of /FPTABLE/ (ANAME2, DNU2, IPARA2).
C
C     Not built here (no Fortran compiler on this build host).  Compile
C     with the reference's flags after radtran_b200.f90, e.g.
C       gfortran -c -fallow-argument-mismatch cirsrtfg_wave_gpu.f
C     from radtran/cirsradg/ (its INCLUDE paths are the reference's),
C     and link the object before cirsradg.a so that it replaces the
C     archive member.
C----------------------------------------------------------------------
      SUBROUTINE cirsrtfg_wave(runname, dist, inormal, iray, fwhm1,
     1  ispace, vwave, nwave, itype1, nem, vem, emissivity, tsurf,
     2  gradtsurf, nv, xmap, vconv, nconv, npath1, calcout,
     3  gradients, iscat)
      USE radtran_b200
      IMPLICIT NONE
      INCLUDE '../includes/arrdef.f'
      INCLUDE '../includes/pathcom.f'
      INCLUDE '../includes/laycom.f'
      INCLUDE '../includes/laygrad.f'
      INCLUDE '../includes/planrad.f'
      INCLUDE '../includes/ciacom.f'
      INCLUDE '../includes/gascom.f'

      CHARACTER*100 runname
      REAL dist, fwhm1, tsurf
      INTEGER inormal, iray, ispace, nwave, itype1, nem, nv, nconv
      INTEGER npath1, iscat
      REAL vwave(nwave), vconv(nconv), vem(maxsec)
      REAL emissivity(maxsec), xmap(maxv,maxgas+2+maxcon,maxpro)
      REAL gradtsurf(maxout3), calcout(maxout3), gradients(maxout4)

C     COMMON blocks the reference's CIRSRTFG_WAVE / CIRSRADG_WAVE read
      INTEGER ilbl
      COMMON /lbltable/ ilbl
      INTEGER idiag, iquiet
      COMMON /diagnostic/ idiag, iquiet
      INTEGER inlte_flag
      REAL nlte_k1, nlte_A
      COMMON /nlte_flags/ inlte_flag, nlte_k1, nlte_A
      REAL swave(maxbin), srad(maxbin), solrad
      INTEGER iread, nspt, iform
      COMMON /solardat/ iread, iform, solrad, swave, srad, nspt

      TYPE(rtb_atm), TARGET, SAVE :: a
      TYPE(rtb_conv), TARGET, SAVE :: cv
      INTEGER(c_int), TARGET, SAVE :: ktab(maxgas)
      INTEGER, PARAMETER :: MFWHM = 1000, MKTA = 100
      REAL, TARGET, SAVE :: vfwhm(MFWHM), xfwhm(MFWHM)
      REAL, TARGET, SAVE :: zheight(maxpro)
      INTEGER nfwhm, i, nkl
      INTEGER(c_int) st, idk(MKTA), isok(MKTA)
      LOGICAL fwhmexist, nlteexist
      CHARACTER*100 fwhmfile, nltefile, klist
      CHARACTER*200 ktafil(MKTA)
      CHARACTER(kind=c_char, len=201), TARGET, SAVE :: cpath(MKTA)
      TYPE(c_ptr) cptr(MKTA)
      INTEGER, SAVE :: loaded = 0

      IF (ilbl .NE. 0) THEN
        PRINT*, 'CIRSRTFG_WAVE (B200): ILBL = ', ilbl,
     1    ' (line-by-line tables) is not on the device path'
        STOP
      ENDIF
      FWHM = fwhm1

C     .fwh: channel-dependent bin width (cirsrtfg_wave.f:182-198)
      nfwhm = 0
      CALL file(runname, fwhmfile, 'fwh')
      INQUIRE(FILE=fwhmfile, EXIST=fwhmexist)
      IF (fwhmexist) THEN
        OPEN(13, FILE=fwhmfile, STATUS='old')
        READ(13,*) nfwhm
        DO i = 1, nfwhm
          READ(13,*) vfwhm(i), xfwhm(i)
        ENDDO
        CLOSE(13)
      ENDIF

C     .lte: non-LTE emission temperatures (cirsrtfg_wave.f:200-213)
      CALL file(runname, nltefile, 'lte')
      INQUIRE(FILE=nltefile, EXIST=nlteexist)
      inlte_flag = 0
      IF (nlteexist) THEN
        OPEN(14, FILE=nltefile, STATUS='old')
        READ(14,*) inlte_flag
        IF (inlte_flag .EQ. 1) READ(14,*) nlte_k1, nlte_A
        CLOSE(14)
      ENDIF

C     layers, paths and gradient matrices: the reference's own set-up
      CALL subpathg(runname)
      npath1 = npath

      CALL rtb_context_open()
      IF (loaded .EQ. 0) THEN
C       the .kta files of <runname>.kls, in order (read_klist.f:88-95)
        CALL file(runname, klist, 'kls')
        OPEN(11, FILE=klist, STATUS='old')
        nkl = 0
 10     READ(11, '(A200)', END=20) ktafil(nkl + 1)
        nkl = nkl + 1
        IF (nkl .LT. MKTA) GOTO 10
 20     CLOSE(11)
        DO i = 1, nkl
          cpath(i) = c_name(ktafil(i))
          cptr(i) = c_loc(cpath(i))
        ENDDO
        st = rtb_load_ktables(ctx, nkl, cptr, idk, isok)
        CALL rtb_check(st, 'rtb_load_ktables')
C       the CIA table that CIAREAD reads (ciaread.f:63-105)
        CALL datarchive(aname1)
        st = rtb_load_cia(ctx, c_name(aname1), dnu1)
        CALL rtb_check(st, 'rtb_load_cia')
        IF (flagh2p .EQ. 1) THEN
          CALL datarchive(aname2)
          st = rtb_load_para_cia(ctx, c_name(aname2), dnu2, ipara2)
          CALL rtb_check(st, 'rtb_load_para_cia')
        ENDIF
        loaded = 1
      ENDIF
C     every gas: the first listed table of its ids covering the
C     wavenumber, per wavenumber, as READ_KLIST assigns lun(iwave,igas)
      DO i = 1, ngas
        ktab(i) = RTB_KTAB_BY_ID
      ENDDO

      a%nlayer = nlayer
      a%ngas = ngas
      a%ncont = ncont
      a%npath = npath
      a%npro = npro
      a%nv = nv
      a%nwave = nwave
      a%ld_lay = maxlay
      a%ld_con = maxcon
      a%ld_v = maxv
      a%ld_param = maxgas + 2 + maxcon
      a%press = c_loc(press)
      a%temp = c_loc(temp)
      a%delh = c_loc(delh)
      a%pp = c_loc(pp)
      a%amount = c_loc(amount)
      a%cont = c_loc(cont)
      a%idgas = c_loc(idgas)
      a%isogas = c_loc(isogas)
      a%ktab = c_loc(ktab)
      a%nlayin = c_loc(nlayin)
      a%imod = c_loc(imod)
      a%layinc = c_loc(layinc)
      a%scale = c_loc(scale)
      a%emtemp = c_loc(emtemp)
      a%dte = c_loc(dte)
      a%dam = c_loc(dam)
      a%dco = c_loc(dco)
      a%dfp = c_loc(dfp)
      a%xmap = c_loc(xmap)
      a%vwave = c_loc(vwave)
C     dust cross sections at vwave: /DUSTSPEC/ interpolated by the
C     caller when ncont > 0 (cirsradg_wave.f:550-575); none here
      a%xsec_ext = c_null_ptr
      a%inormal = inormal
      a%iray = iray
      a%itype = itype1
      a%ispace = ispace
      a%flagh2p = flagh2p
      a%ilbl = ilbl
      a%inlte = inlte_flag
      a%iform = iform
      a%tsurf = tsurf
      a%fwhm = fwhm1
      a%nem = nem
      a%vem = c_loc(vem)
      a%emissivity = c_loc(emissivity)
      a%hfp = c_loc(hfp)
C     RADIUS1 and radextra as cirsrtfg_wave.f:380-388 set them
      a%radius1 = radius2
      a%radextra = 0.0
      IF (ipzen .EQ. 2) THEN
        CALL readprfheight(runname, npro, zheight)
        a%radextra = zheight(npro)
      ENDIF
      a%nlte_k1 = nlte_k1
      a%nlte_A = nlte_A
      a%dist = dist
      a%ih2o = ih2o
      a%ich4 = ich4
      a%inh3 = inh3
      a%io3 = io3
      a%iuvscat = iuvscat
C     the channels: vconv, the .fwh widths when present; a .fil filter
C     set (FWHM < 0) is read with rtb_read_fil into vcen/nsub/vfil/fil
      cv%nconv = nconv
      cv%vconv = c_loc(vconv)
      cv%nfwhm = nfwhm
      cv%vfwhm = c_loc(vfwhm)
      cv%xfwhm = c_loc(xfwhm)
      cv%nfil = 0
      cv%vcen = c_null_ptr
      cv%nsub = c_null_ptr
      cv%vfil = c_null_ptr
      cv%fil = c_null_ptr
      a%conv = c_loc(cv)

      st = rtb_cirsrtfg_wave(ctx, a, calcout, gradients, gradtsurf)
      CALL rtb_check(st, 'CIRSRTFG_WAVE')
      RETURN
      END
