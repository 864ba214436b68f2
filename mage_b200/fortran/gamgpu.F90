! ISO_C_BINDING interface of libgamgpu.so (include/gamgpu.h) for the Fortran
! driver of GAMERA. The host arrays are the driver's own State_T / Grid_T
! allocatables, passed with c_loc: column-major, ghosts included, no copies.
!
! Intended caller: gamApp_T%AdvanceModel (gamtypessub.F90:74-90), which uploads
! State/oState, calls gam_advance_model and downloads the new State.
module gamgpu
    use, intrinsic :: iso_c_binding
    implicit none

    integer(c_int), parameter :: GAM_OK = 0, GAM_EINVAL = 1, GAM_EBADDIM = 2, GAM_ECUDA = 3, &
                                 GAM_EDT_BAD = 4, GAM_EDT_DISASTER = 5, GAM_ESTATE = 6, GAM_EHOOK = 7, &
                                 GAM_EBOUNDS = 8
    integer(c_int), parameter :: GAM_BC_PERIODIC = 0, GAM_BC_NONE = 1, GAM_BC_ZEROGRAD = 2, GAM_BC_SPHIN = 3, &
                                 GAM_BC_WIND = 4, GAM_BC_HALO = 5, GAM_BC_INFLOW = 6, &
                                 GAM_BC_ION = 7, GAM_BC_LFM = 8
    integer(c_int), parameter :: GAM_RECON_8CENT = 0, GAM_RECON_7UP = 1
    integer(c_int), parameter :: GAM_FP64 = 0, GAM_FP32 = 1

    type, bind(C) :: gam_params
        integer(c_int32_t) :: Nip, Njp, Nkp, nG
        real(c_double) :: gamma, CFL, pdmb, Vd0, cHogH, cHogM, dFloor, pFloor
        real(c_double) :: tFin, dt0, limDT0, fixedTimestep
        integer(c_int32_t) :: rmeth, doLFMLim, doMHD, doBackground, do25D, precision, strict
        integer(c_int32_t) :: bc(6)
        integer(c_int32_t) :: doBoris
        real(c_double) :: Ca
        integer(c_int32_t) :: doAB3
    end type gam_params

    ! inflow and wind values and wind tables of the differentiation form's
    ! I-side boundaries (device pointers in the form's precision)
    type, bind(C) :: gam_iside
        real(c_double) :: inflow(8), wind(8)
        type(c_ptr) :: wC, wF(3), sF(3)
    end type gam_iside

    interface
        integer(c_int) function gam_default_params(p, Nip, Njp, Nkp) bind(C, name="gam_default_params")
            import :: c_int, c_int32_t, gam_params
            type(gam_params), intent(out) :: p
            integer(c_int32_t), value :: Nip, Njp, Nkp
        end function
        integer(c_int) function gam_create(p, h) bind(C, name="gam_create")
            import :: c_int, c_ptr, gam_params
            type(gam_params), intent(in) :: p
            type(c_ptr), intent(out) :: h
        end function
        integer(c_int) function gam_destroy(h) bind(C, name="gam_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function
        type(c_ptr) function gam_last_error(h) bind(C, name="gam_last_error")
            import :: c_ptr
            type(c_ptr), value :: h
        end function
        integer(c_int) function gam_set_geometry(h, xyz) bind(C, name="gam_set_geometry")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, xyz
        end function
        integer(c_int) function gam_set_geometry_arrays(h, face, xfc, Tf, volume, xyzcc, di, dj, dk, edge, Te, Teb) &
                bind(C, name="gam_set_geometry_arrays")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, face, xfc, Tf, volume, xyzcc, di, dj, dk, edge, Te, Teb
        end function
        integer(c_int) function gam_upload_state(h, Gas, magFlux, Bxyz, oGas, omagFlux, time, otime, dt, ts) &
                bind(C, name="gam_upload_state")
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: h, Gas, magFlux, Bxyz, oGas, omagFlux
            real(c_double), value :: time, otime, dt
            integer(c_int32_t), value :: ts
        end function
        integer(c_int) function gam_download_state(h, Gas, magFlux, Bxyz, oGas, omagFlux, time, otime, dt, ts) &
                bind(C, name="gam_download_state")
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: h, Gas, magFlux, Bxyz, oGas, omagFlux
            real(c_double), intent(out) :: time, otime, dt
            integer(c_int32_t), intent(out) :: ts
        end function
        integer(c_int) function gam_step(h, nsteps, dt, t) bind(C, name="gam_step")
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: nsteps
            real(c_double), intent(out) :: dt, t
        end function
        integer(c_int) function gam_advance_model(h, dt, t) bind(C, name="gam_advance_model")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), value :: dt
            real(c_double), intent(out) :: t
        end function
        integer(c_int) function gam_calc_dt(h, dt) bind(C, name="gam_calc_dt")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: dt
        end function
        integer(c_int) function gam_divb(h, total) bind(C, name="gam_divb")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: total
        end function
        integer(c_int) function gam_totals(h, out) bind(C, name="gam_totals")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: out(5)
        end function
        integer(c_int) function gam_set_background(h, fcB0, bFlux0, edgB0, B0, dpB0) bind(C, name="gam_set_background")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, fcB0, bFlux0, edgB0, B0, dpB0
        end function
        integer(c_int) function gam_get_background(h, fcB0, bFlux0, edgB0, B0, dpB0) bind(C, name="gam_get_background")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, fcB0, bFlux0, edgB0, B0, dpB0
        end function
        integer(c_int) function gam_set_background_dipole(h, M0) bind(C, name="gam_set_background_dipole")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), value :: M0
        end function
        integer(c_int) function gam_set_wind(h, wind) bind(C, name="gam_set_wind")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: wind(8)
        end function
        ! solar-wind time series: t(n), rho(n), P(n), V(3,n), B(3,n), xyzBS(3,n) or c_null_ptr
        integer(c_int) function gam_set_wind_series(h, n, t, rho, P, V, B, xyzBS, Bx0, ByC, BzC) &
                bind(C, name="gam_set_wind_series")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t), value :: n
            real(c_double), intent(in) :: t(*), rho(*), P(*), V(*), B(*)
            type(c_ptr), value :: xyzBS
            real(c_double), value :: Bx0, ByC, BzC
        end function
        ! the reference's test problems: which = 2 ADV1D, 3 ADV2D, 4 LOOP2D, 5 ALFVEN
        integer(c_int) function gam_init_test_problem(h, which, a, b) bind(C, name="gam_init_test_problem")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t), value :: which
            real(c_double), value :: a, b
        end function
        integer(c_int) function gam_set_inflow(h, state) bind(C, name="gam_set_inflow")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: state(8)
        end function
        ! record of the bounds-check build (libgamgpu_check.so); fired = -1 without checks
        integer(c_int) function gam_bounds_status(h, fired, kernel, index) bind(C, name="gam_bounds_status")
            import :: c_int, c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: h
            integer(c_int32_t), intent(out) :: fired, kernel
            integer(c_int64_t), intent(out) :: index
        end function
        ! ooState of the AB3 predictor (doAB3): magFlux(isg:ieg+1,jsg:jeg+1,ksg:keg+1,1:3) and time
        integer(c_int) function gam_set_oostate(h, oomagFlux, ootime) bind(C, name="gam_set_oostate")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: oomagFlux(*)
            real(c_double), value :: ootime
        end function
        integer(c_int) function gam_get_oostate(h, oomagFlux, ootime) bind(C, name="gam_get_oostate")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: oomagFlux(*)
            real(c_double), intent(out) :: ootime
        end function
        ! tiling: the MPI driver (gamAppMpi_T) packs/unpacks halos in device
        ! buffers, direction by direction (I, J, K), and reduces dt between
        ! gam_step_begin and gam_step_end; the gam_halo_* forms are dir = 2
        integer(c_int) function gam_set_tile_edges(h, dir, lowest, highest) bind(C, name="gam_set_tile_edges")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: dir, lowest, highest
        end function
        integer(c_int) function gam_tile_halo_bytes(h, dir, nbytes) bind(C, name="gam_tile_halo_bytes")
            import :: c_int, c_ptr, c_int32_t, c_int64_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: dir
            integer(c_int64_t), intent(out) :: nbytes
        end function
        integer(c_int) function gam_tile_halo_pack(h, dir, side, dev_buf) bind(C, name="gam_tile_halo_pack")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h, dev_buf
            integer(c_int32_t), value :: dir, side
        end function
        integer(c_int) function gam_tile_halo_unpack(h, dir, side, dev_buf, copyB) &
                bind(C, name="gam_tile_halo_unpack")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h, dev_buf
            integer(c_int32_t), value :: dir, side, copyB
        end function
        integer(c_int) function gam_set_slab_edges(h, lowest, highest) bind(C, name="gam_set_slab_edges")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: lowest, highest
        end function
        integer(c_int) function gam_halo_bytes(h, nbytes) bind(C, name="gam_halo_bytes")
            import :: c_int, c_ptr, c_int64_t
            type(c_ptr), value :: h
            integer(c_int64_t), intent(out) :: nbytes
        end function
        integer(c_int) function gam_halo_pack(h, side, dev_buf) bind(C, name="gam_halo_pack")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h, dev_buf
            integer(c_int32_t), value :: side
        end function
        integer(c_int) function gam_halo_unpack(h, side, dev_buf, copyB) bind(C, name="gam_halo_unpack")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h, dev_buf
            integer(c_int32_t), value :: side, copyB
        end function
        integer(c_int) function gam_init_finish_halo(h, dt) bind(C, name="gam_init_finish_halo")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: dt
        end function
        integer(c_int) function gam_set_start(h, dt) bind(C, name="gam_set_start")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), value :: dt
        end function
        integer(c_int) function gam_step_begin(h) bind(C, name="gam_step_begin")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function
        integer(c_int) function gam_dt_partial(h, bits, nbad) bind(C, name="gam_dt_partial")
            import :: c_int, c_ptr, c_int64_t, c_int32_t
            type(c_ptr), value :: h
            integer(c_int64_t), intent(out) :: bits
            integer(c_int32_t), intent(out) :: nbad
        end function
        integer(c_int) function gam_step_end(h, bits, nbad, dt, t) bind(C, name="gam_step_end")
            import :: c_int, c_ptr, c_int64_t, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int64_t), value :: bits
            integer(c_int32_t), value :: nbad
            real(c_double), intent(out) :: dt, t
        end function
        ! the same step with the dt reduction on the device: bits and nbad are
        ! device addresses (c_devptr of CUDA Fortran, or c_ptr of a device
        ! buffer) of one int64 each; stream is a cudaStream_t
        integer(c_int) function gam_set_stream(h, stream) bind(C, name="gam_set_stream")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, stream
        end function
        integer(c_int) function gam_step_begin_dev(h) bind(C, name="gam_step_begin_dev")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function
        integer(c_int) function gam_dt_partial_dev(h, bits, nbad) bind(C, name="gam_dt_partial_dev")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, bits, nbad
        end function
        integer(c_int) function gam_step_end_dev(h, bits, nbad) bind(C, name="gam_step_end_dev")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, bits, nbad
        end function
        integer(c_int) function gam_step_status(h, dt, t) bind(C, name="gam_step_status")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: dt, t
        end function
        integer(c_int) function gam_get_geometry_arrays(h, face, xfc, Tf, volume, xyzcc, di, dj, dk, edge, Te, Teb) &
                bind(C, name="gam_get_geometry_arrays")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, face, xfc, Tf, volume, xyzcc, di, dj, dk, edge, Te, Teb
        end function
        integer(c_int) function gam_init_orszag_tang(h) bind(C, name="gam_init_orszag_tang")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function
        integer(c_int) function gam_init_blast_wave(h, bw) bind(C, name="gam_init_blast_wave")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: bw(9)
        end function
        integer(c_int) function gam_profile_step(h, reps, ms, n) bind(C, name="gam_profile_step")
            import :: c_int, c_ptr, c_int32_t, c_double
            type(c_ptr), value :: h
            integer(c_int32_t), value :: reps, n
            real(c_double), intent(out) :: ms(n)
        end function
        integer(c_int) function gam_last_step_ms(h, ms) bind(C, name="gam_last_step_ms")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: ms
        end function
        integer(c_int) function gam_totals_noalloc(Gas, volume, Nip, Njp, Nkp, out, stream, err, errlen) &
                bind(C, name="gam_totals_noalloc")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: Gas, volume, out, stream, err
            integer(c_int32_t), value :: Nip, Njp, Nkp, errlen
        end function
        ! differentiation form: stage forwards and their hand-written adjoints on
        ! device arrays (see include/gamgpu.h for the layouts)
        integer(c_int) function gam_flux_forward(p, fp32, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, gF, mF, &
                stream) bind(C, name="gam_flux_forward")
            import :: c_int, c_ptr, c_int32_t, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), value :: QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, gF, mF, stream
        end function
        integer(c_int) function gam_flux_adjoint(p, fp32, QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, dgF, &
                dmF, dQW, dWn, dQB, dBlim, dBnf, stream) bind(C, name="gam_flux_adjoint")
            import :: c_int, c_ptr, c_int32_t, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), value :: QW, Wn, QB, Blim, Bnf, volume, face, Tf, fcB0, bFlux0, dgF, dmF, dQW, dWn, dQB, dBlim, &
                                  dBnf, stream
        end function
        integer(c_int) function gam_efield_forward(p, fp32, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, &
                E, stream) bind(C, name="gam_efield_forward")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), value :: Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, AVf, E, stream
            real(c_double), value :: dt
        end function
        integer(c_int) function gam_efield_adjoint(p, fp32, Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, dt, AVf, &
                dE, dDh, dabh, dbn, dVdV, dAVf, stream) bind(C, name="gam_efield_adjoint")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), value :: Dh, abh, bn, VdV, volume, face, edge, Te, Teb, edgB0, AVf, dE, dDh, dabh, dbn, dVdV, dAVf, &
                                  stream
            real(c_double), value :: dt
        end function
        integer(c_int) function gam_predict_stage(p, fp32, st, geo, pdt, odt, out, din, aB, dst, stream) &
                bind(C, name="gam_predict_stage")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), intent(in) :: st(4), geo(5)
            real(c_double), value :: pdt, odt
            type(c_ptr), value :: out, din, aB, dst, stream
        end function
        integer(c_int) function gam_update_stage(p, fp32, in, geo, dpB0, dt, out, din, sU, sM, dst, stream) &
                bind(C, name="gam_update_stage")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), intent(in) :: in(5), geo(4)
            type(c_ptr), value :: dpB0, out, din, sU, sM, dst, stream
            real(c_double), value :: dt
        end function
        integer(c_int) function gam_step_work_bytes(p, fp32, bytes) bind(C, name="gam_step_work_bytes")
            import :: c_int, c_int32_t, c_int64_t, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            integer(c_int64_t), intent(out) :: bytes
        end function
        integer(c_int) function gam_step_fwd_save(p, fp32, geo, bg, st, dt, odt, nxt, work, stream) &
                bind(C, name="gam_step_fwd_save")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), intent(in) :: geo(9), st(4), nxt(3)
            type(c_ptr), value :: bg, work, stream
            real(c_double), value :: dt, odt
        end function
        integer(c_int) function gam_step_adj(p, fp32, geo, bg, st, dt, odt, saved, dnxt, dst, work, stream) &
                bind(C, name="gam_step_adj")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32, saved
            type(c_ptr), intent(in) :: geo(9), st(4), dnxt(3), dst(4)
            type(c_ptr), value :: bg, work, stream
            real(c_double), value :: dt, odt
        end function
        ! ring averaging about the LFM axis, before the geometry
        integer(c_int) function gam_set_rings(h, NumR, Nch, recon, NFTmag, doClean, doFastClean) &
                bind(C, name="gam_set_rings")
            import :: c_int, c_ptr, c_int32_t
            type(c_ptr), value :: h
            integer(c_int32_t), value :: NumR, recon, NFTmag, doClean, doFastClean
            integer(c_int32_t), intent(in) :: Nch(*)
        end function
        integer(c_int) function gam_ring_defaults(Np, aggressive, NumR, Nch) bind(C, name="gam_ring_defaults")
            import :: c_int, c_int32_t
            integer(c_int32_t), value :: Np, aggressive
            integer(c_int32_t), intent(out) :: NumR, Nch(32)
        end function
        ! a tile away from the inner boundary leaves out both fields (NULL)
        integer(c_int) function gam_set_ionosphere(h, inExyz, inEijk, M0, dtCpl, doIonPush, nIonP, dtSW0) &
                bind(C, name="gam_set_ionosphere")
            import :: c_int, c_ptr, c_double, c_int32_t
            type(c_ptr), value :: h
            real(c_double), intent(in), optional :: inExyz(*), inEijk(*)
            real(c_double), value :: M0, dtCpl, dtSW0
            integer(c_int32_t), value :: doIonPush, nIonP
        end function
        integer(c_int) function gam_iside_fill(p, fp32, geo, is, B, Gas, mf, stream) &
                bind(C, name="gam_iside_fill")
            import :: c_int, c_ptr, c_int32_t, gam_params, gam_iside
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), intent(in) :: geo(2)
            type(gam_iside), intent(in) :: is
            type(c_ptr), value :: B, Gas, mf, stream
        end function
        integer(c_int) function gam_iside_adjoint(p, fp32, geo, is, Gas, B, dGas, dMf, dB, dinflow, stream) &
                bind(C, name="gam_iside_adjoint")
            import :: c_int, c_ptr, c_int32_t, gam_params, gam_iside
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), intent(in) :: geo(2)
            type(gam_iside), intent(in) :: is
            type(c_ptr), value :: Gas, B, dGas, dMf, dB, dinflow, stream
        end function
        integer(c_int) function gam_step_fwd_save_iside(p, fp32, geo, bg, is, st, dt, odt, nxt, work, stream) &
                bind(C, name="gam_step_fwd_save_iside")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params, gam_iside
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32
            type(c_ptr), intent(in) :: geo(9), st(4), nxt(3)
            type(gam_iside), intent(in) :: is
            type(c_ptr), value :: bg, work, stream
            real(c_double), value :: dt, odt
        end function
        integer(c_int) function gam_step_adj_iside(p, fp32, geo, bg, is, st, dt, odt, saved, dnxt, dst, dinflow, &
                                                   work, stream) bind(C, name="gam_step_adj_iside")
            import :: c_int, c_ptr, c_int32_t, c_double, gam_params, gam_iside
            type(gam_params), intent(in) :: p
            integer(c_int32_t), value :: fp32, saved
            type(c_ptr), intent(in) :: geo(9), st(4), dnxt(3), dst(4)
            type(gam_iside), intent(in) :: is
            type(c_ptr), value :: bg, dinflow, work, stream
            real(c_double), value :: dt, odt
        end function
        integer(c_int) function gam_write_restart(h, path) bind(C, name="gam_write_restart")
            import :: c_int, c_ptr, c_char
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: path(*)
        end function
        integer(c_int) function gam_read_restart(h, path) bind(C, name="gam_read_restart")
            import :: c_int, c_ptr, c_char
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: path(*)
        end function
        integer(c_int) function gam_init_dipole_wind(h, wind, seed, amp) bind(C, name="gam_init_dipole_wind")
            import :: c_int, c_ptr, c_double, c_int64_t
            type(c_ptr), value :: h
            real(c_double), intent(in) :: wind(8)
            integer(c_int64_t), value :: seed
            real(c_double), value :: amp
        end function
    end interface

contains

    !> Error text of the last failed call on h, as a Fortran string.
    function gam_error_string(h) result(msg)
        type(c_ptr), intent(in) :: h
        character(len=256) :: msg
        character(kind=c_char), pointer :: cs(:)
        integer :: n
        msg = ""
        call c_f_pointer(gam_last_error(h), cs, [256])
        do n = 1, 256
            if (cs(n) == c_null_char) exit
            msg(n:n) = cs(n)
        enddo
    end function gam_error_string

end module gamgpu
