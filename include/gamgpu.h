/* gamgpu.h -- C ABI of the B200 GAMERA MHD step.
 *
 * The entry points replace the CPU time step of the reference's GAMERA solver
 * (Kaiju/MAGE, Fortran) for a single-domain grid. Fortran callers bind them
 * with ISO_C_BINDING (module gamgpu, mage_b200/fortran/gamgpu.F90); Python
 * binds them with ctypes (mage_b200/gamera.py).
 *
 * Conventions
 *  - Every entry point returns an int status, GAM_OK (0) on success. On error
 *    gam_last_error(h) returns a message; the handle stays usable.
 *  - Host arrays are the reference's own Fortran arrays, passed by c_loc:
 *    column-major, i fastest, including the nG = 4 ghost layers.
 *      cell arrays  A(isg:ieg,   jsg:jeg,   ksg:keg,   1:nc)
 *      face arrays  A(isg:ieg+1, jsg:jeg+1, ksg:keg+1, 1:nc)
 *    with isg = 1-nG, ieg = Nip+nG (likewise j, k). No pointer is retained
 *    past a call.
 *  - One handle per host thread; calls on a handle are serialised on the
 *    handle's CUDA stream. Handles are independent of each other.
 */
#ifndef GAMGPU_H
#define GAMGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    GAM_OK = 0,
    GAM_EINVAL = 1,        /* bad argument / unsupported option            */
    GAM_EBADDIM = 2,       /* Nip%8 != 0 or Nip < 16 (init.F90:817-826)    */
    GAM_ECUDA = 3,         /* CUDA runtime error                           */
    GAM_EDT_BAD = 4,       /* dt dropped 10x or below limDT0 (step.F90:111-128) */
    GAM_EDT_DISASTER = 5,  /* dt <= TINY or no finite dt (step.F90:102-105,131-134) */
    GAM_ESTATE = 6,        /* call out of order (e.g. step before geometry) */
    GAM_EHOOK = 7,         /* a Model%Hack* hook is set: not supported on the GPU */
    GAM_EBOUNDS = 8        /* bounds-check build only: a kernel's index check failed */
};

/* Boundary kinds (EnforceBCs, step.F90:17-55). Per side: INI periodic, none,
 * GAM_BC_SPHIN (bcs.F90:934-957) or GAM_BC_INFLOW; OUTI periodic, none,
 * GAM_BC_WIND (constant solar wind, apps/wind.F90:206-391) or GAM_BC_ZEROGRAD
 * (zeroGrad_obcI, bcs.F90:820-850); INJ/OUTJ periodic, none or
 * GAM_BC_ZEROGRAD (bcs.F90:853-892); INK/OUTK periodic or none. Any side of
 * a tile may be GAM_BC_HALO instead (filled by the caller's halo exchange).
 * GAM_BC_INFLOW has no counterpart in the reference: the 4 inner-I ghost
 * layers hold a uniform state (gam_set_inflow) and the face fluxes of its
 * field, the shape of zeroGrad_obcI with a given state in place of the last
 * active cell. GAM_BC_ION (inner I) is the ionospheric boundary of the
 * magnetosphere (IonInnerBC_T, voltron/ICs/earthcmi.F90:441-583) together
 * with the model hooks that come with it (gam_set_ionosphere). */
enum { GAM_BC_PERIODIC = 0, GAM_BC_NONE = 1, GAM_BC_ZEROGRAD = 2, GAM_BC_SPHIN = 3, GAM_BC_WIND = 4,
       GAM_BC_HALO = 5 /* a tile's side towards a neighbour: filled by the caller's halo exchange */,
       GAM_BC_INFLOW = 6, GAM_BC_ION = 7,
       GAM_BC_LFM = 8 /* INJ / OUTJ on the LFM axis (lfmIn / lfmOut, bcs.F90:1019-1106), with rings */ };
enum { GAM_RECON_8CENT = 0, GAM_RECON_7UP = 1 };
enum { GAM_FP64 = 0, GAM_FP32 = 1 };

/* Model keys of the step. Defaults of the reference (init.F90:312-484):
 * gamma 5/3, pdmb 0.75, CFL min(0.5/(pdmb+0.5),0.3), Vd0 0.5, cHogH = cHogM
 * = 0.25, floors 1e-12, rmeth 8CENT, lfmlim T, limDT0 1e-3. */
typedef struct gam_params {
    int32_t Nip, Njp, Nkp;  /* active cells per direction                  */
    int32_t nG;             /* ghost layers; must be 4                       */
    double gamma, CFL, pdmb, Vd0, cHogH, cHogM, dFloor, pFloor;
    double tFin;            /* Model%tFin: dt is clamped to land on it       */
    double dt0;             /* Model%dt0: 0 disables the dt0-based checks    */
    double limDT0;          /* Model%limDT0                                  */
    double fixedTimestep;   /* > 0: Model%fixedTimestep with this dt         */
    int32_t rmeth;          /* GAM_RECON_8CENT or GAM_RECON_7UP              */
    int32_t doLFMLim, doMHD, doBackground, do25D;
    int32_t precision;      /* GAM_FP64 (drop-in) or GAM_FP32 (bulk FP32)    */
    int32_t strict;         /* 1: kernels without FMA contraction            */
    int32_t bc[6];          /* INI, OUTI, INJ, OUTJ, INK, OUTK: GAM_BC_*     */
    int32_t doBoris;        /* physics/doBoris (init.F90:417-423): Boris-limited
                               Alfven speed, Boris hogs and the nuclear option in
                               the fluxes, CellBoris in the update */
    double Ca;              /* physics/Ca, the Boris speed of light (code units) */
    int32_t doAB3;          /* sim/doAB3 (init.F90:377): AB3 predictor with ooState
                               (mhdgroup.F90:444-517, 721-731) */
} gam_params;

typedef struct gam_handle gam_handle;

/* Fill p with the reference defaults for an Nip x Njp x Nkp grid. */
int gam_default_params(gam_params* p, int32_t Nip, int32_t Njp, int32_t Nkp);

/* Replaces Hatch/initSolver allocation (init.F90:38-59, 486-509). */
int gam_create(const gam_params* p, gam_handle** out);
int gam_destroy(gam_handle* h);
const char* gam_last_error(gam_handle* h);

/* Corner coordinates xyz(isg:ieg+1,jsg:jeg+1,ksg:keg+1,1:3). The FP64 metric
 * (face areas/centroids/triads, volumes, barycentres, CFL lengths, edge
 * lengths/triads, edge B maps) is computed on the GPU.
 * Replaces Corners2Grid + ebGeom (init.F90:793-1137). */
int gam_set_geometry(gam_handle* h, const double* xyz);

/* The Fortran-precomputed Grid_T arrays (gamtypes.F90:168-250), as an
 * alternative to gam_set_geometry for drivers that already hold them:
 * face(f,3) xfc(f,3,3) Tf(f,9,3) volume(c) xyzcc(c,3) di,dj,dk(c)
 * edge(f,3) Te(f,9,3) Teb(f,4,3); f = face-sized, c = cell-sized. */
int gam_set_geometry_arrays(gam_handle* h, const double* face, const double* xfc, const double* Tf,
                            const double* volume, const double* xyzcc, const double* di, const double* dj,
                            const double* dk, const double* edge, const double* Te, const double* Teb);

/* Copy back the metric (same layout as gam_set_geometry_arrays). */
int gam_get_geometry_arrays(gam_handle* h, double* face, double* xfc, double* Tf, double* volume, double* xyzcc,
                            double* di, double* dj, double* dk, double* edge, double* Te, double* Teb);

/* State%Gas(c,5), State%magFlux(f,3), State%Bxyz(c,3) and the previous state
 * oState%Gas, oState%magFlux, with State%time, oState%time, Model%dt and
 * Model%ts. Replaces the in-memory state of gamApp_T (gamtypes.F90:301-321).
 * oGas = omagFlux = NULL (after a first full upload): oState stays as it is
 * on the device and only State crosses PCIe. After gam_step the device's
 * oState is the State before that step (CopyState, mhdgroup.F90:202-256),
 * i.e. the oState of a driver that steps one AdvanceModel at a time.
 * Bxyz = NULL: State%Bxyz is computed on the device from the uploaded fluxes
 * (bFlux2Fld, gridutils.F90:281-301, which every step and the
 * initialisation end with), so only Gas and magFlux cross PCIe. */
int gam_upload_state(gam_handle* h, const double* Gas, const double* magFlux, const double* Bxyz,
                     const double* oGas, const double* omagFlux, double time, double otime, double dt, int32_t ts);
int gam_download_state(gam_handle* h, double* Gas, double* magFlux, double* Bxyz, double* oGas,
                       double* omagFlux, double* time, double* otime, double* dt, int32_t* ts);

/* nsteps x stepGamera (gamapp.F90:73-91): AdvanceMHD, t += dt, CalcDT,
 * EnforceBCs, bFlux2Fld. On return *dt and *t hold Model%dt and Model%t.
 * A failed CalcDT stops the sequence with GAM_EDT_BAD / GAM_EDT_DISASTER and
 * leaves the state as the reference leaves it when it stops (after the
 * update, before the boundary conditions). */
int gam_step(gam_handle* h, int32_t nsteps, double* dt, double* t);

/* CalcDT on the current state (step.F90:58-168), without changing Model%dt. */
int gam_calc_dt(gam_handle* h, double* dt);

/* Sum over active cells of |div B| (gridutils.F90:717-770). */
int gam_divb(gam_handle* h, double* total);

/* Volume-weighted totals over active cells of the five conserved variables
 * (mass, momentum x/y/z, energy), FP64 deterministic tree reduction. */
int gam_totals(gam_handle* h, double out[5]);

/* Wall time of the last gam_step call measured with CUDA events (ms). */
int gam_last_step_ms(gam_handle* h, double* ms);

/* Diagnostic: device time (ms) of each kernel of one step, averaged over
 * reps repeated launches on the current state, in step order: ms[0] begin,
 * [1] predictor, [2..7] Mom2Face/VxB for E_i, E_j, E_k, [8..10] fluxes i/j/k,
 * [11] face update, [12] cell update + dt, [13] dt decision, [14] boundary
 * fill (n >= 15). The state is left as it was. */
int gam_profile_step(gam_handle* h, int32_t reps, double* ms, int32_t n);

/* gamApp_T%AdvanceModel(dt) (gamtypessub.F90:74-90): one step, then steps
 * while Model%t < t_start + dt. */
int gam_advance_model(gam_handle* h, double dt, double* t_out);

/* Problem set-up on the device from the metric already set, then the
 * reference's initialisation order (init.F90:190-246): Bxyz, first boundary
 * conditions, oState = State, first CalcDT, oState%time = t - dt.
 *   gam_init_orszag_tang: initOT2D (prob.F90:74-119)
 *   gam_init_blast_wave : initBW (prob.F90:190-298), vector-potential field;
 *     bw = {x0, y0, z0, D0, P0, pRat, dRat, rC, B0}; needs gam_set_geometry. */
int gam_init_orszag_tang(gam_handle* h);
int gam_init_blast_wave(gam_handle* h, const double bw[9]);

/* Background field (doBackground = 1; Grid_T fcB0, bFlux0, edgB0, B0, dpB0,
 * gamtypes.F90:233-242). All five are cell-sized Fortran arrays with ghosts:
 * fcB0(.., 3, 3) (component, face), bFlux0(.., 3), edgB0(.., 2, 3), B0(.., 3),
 * dpB0(.., 3).
 *   gam_set_background       : the driver's own arrays, as AddB0 left them
 *                              (background.F90:20-167)
 *   gam_get_background       : copy back (any pointer may be NULL)
 *   gam_set_background_dipole: AddB0 on the device for the dipole field of
 *                              moment (0, 0, M0) (msphutils.F90:534-551);
 *                              needs gam_set_geometry */
int gam_set_background(gam_handle* h, const double* fcB0, const double* bFlux0, const double* edgB0,
                       const double* B0, const double* dpB0);
int gam_get_background(gam_handle* h, double* fcB0, double* bFlux0, double* edgB0, double* B0, double* dpB0);
int gam_set_background_dipole(gam_handle* h, double M0);

/* The reference's test problems (src/gamera/prob.F90) as initial conditions,
 * then the initialisation order of gam_init_orszag_tang:
 *   GAM_IC_ADV1D   initADV1D (:671-736), four shapes advected at speed 1
 *                  (the reference sets gamma 1.4 for it: pass it in gam_params)
 *   GAM_IC_ADV2D   initADV2D (:739-797), a = V0, b = alpha (degrees)
 *   GAM_IC_LOOP2D  initLoop (:436-500), a = V0, b = alpha (degrees)
 *   GAM_IC_ALFVEN  initALFVEN (:1027-1083), a = alp (radians)
 * with the other prob/ keys at the reference's defaults. Needs gam_set_geometry. */
enum { GAM_IC_ADV1D = 2, GAM_IC_ADV2D = 3, GAM_IC_LOOP2D = 4, GAM_IC_ALFVEN = 5 };
int gam_init_test_problem(gam_handle* h, int32_t which, double a, double b);

/* Solar-wind state of the outer-I boundary (bc[1] = GAM_BC_WIND), constant in
 * space and time: wind = {rho, P, Vx, Vy, Vz, Bx, By, Bz}. The blend weights
 * (wgtWind, apps/wind.F90:180-203) and the wind face fluxes of the ghost
 * layers are computed here once from the metric. Replaces the windBC_T set-up
 * of the driver (apps/wind.F90:40-176) for a constant wind. */
int gam_set_wind(gam_handle* h, const double wind[8]);

/* A solar-wind time series for the outer-I wind boundary (bc[1] = GAM_BC_WIND)
 * in place of the constant wind: n >= 2 rows at uniformly spaced times t
 * (readWind's check, apps/wind.F90:691-699) of density, pressure, velocity
 * V[3*r+x] and field B[3*r+x], in code units (the driver converts its file as
 * readWind does, :655-668); xyzBS[3*r+x] the bow-shock marker (NULL: the
 * origin); Bx0, ByC, BzC the tilted-front coefficients (Bx = Bx0 + ByC*By +
 * BzC*Bz replaces the series' Bx, :720-727). Each boundary fill takes the
 * wind at every ghost cell and face at its lag time along the front
 * (RefreshWind, GetWindAt, wgtWind, :116-203; InterpWind and InterpWgts,
 * :766-868, with the reference's doWindInterp = F: the row at or below the
 * time; a null field before the first row, no spin-up sequence). The weights
 * use CUDA's acos and exp. With doBoris a series faster than Ca is refused
 * (:744-750). The initial condition still comes from gam_init_dipole_wind's
 * constant state; call this after it. */
int gam_set_wind_series(gam_handle* h, int32_t n, const double* t, const double* rho, const double* P,
                        const double* V, const double* B, const double* xyzBS, double Bx0, double ByC, double BzC);

/* State of the uniform inner-I inflow (bc[0] = GAM_BC_INFLOW), same order as
 * the wind: {rho, P, Vx, Vy, Vz, Bx, By, Bz}. Ghost cell is-n (n = 1..4, every
 * j, k of the cell ranges) gets the conserved form of that state (CellP2C,
 * gamutils.F90:362-383), its I face is-n and its J and K faces the flux
 * face * (n . B), and, in the first boundary fill only, its Bxyz from those
 * fluxes (steps recompute every ghost's Bxyz). Call before the initial
 * condition; calling it later changes the boundary from the next step on. */
int gam_set_inflow(gam_handle* h, const double state[8]);

/* The ionospheric inner boundary (bc[0] = GAM_BC_ION) and the per-step model
 * hooks of the reference's magnetosphere set-up that act on it
 * (voltron/ICs/earthcmi.F90 with its defaults: IonInnerBC_T, EFix, PerStep):
 *   - the boundary (IonInner :441-583, CellPlasmaBC msphingest.F90:268-372,
 *     single fluid, no ingestion): ghost cell is-n takes the density and
 *     pressure of its mirror cell is+n-1 (k wrapped into the active range)
 *     and the E x B velocity of the coupling field inExyz(5-n) in the dipole
 *     field at its centre, perpendicular to the radius, with only the inward
 *     part of its radial component; its faces take zero flux;
 *   - HackE (EFix :321-354): IonEFix (msphutils.F90:214-240), the J and K
 *     EMFs of the first shell from the coupling field inEijk(5), then
 *     FixEFieldLFM (gamdebug.F90:149-175), the I and J EMFs of the two
 *     periodic k ends set to their mean;
 *   - HackStep (PerStep :224-263): PushIon (:586-663), which moves the
 *     velocity of the first nIonP active shells towards the E x B velocity at
 *     the rate dt / (shell * dtCpl), before CalcDT;
 *   - with the solar wind outside (bc[1] = GAM_BC_WIND, the constant wind of
 *     gam_set_wind): WindEFix (apps/wind.F90:489-566), the EMFs of the outer
 *     4 shells blended with the wind's -V x B by the wind weight at each
 *     edge centre, plus DiffuseOuter (:570-616) on the outermost, between
 *     IonEFix and FixEFieldLFM; NudgeSW (:394-486), the last active cell
 *     nudged towards the wind over max(dtSW0 / weight, dt), after PushIon.
 * inExyz is the Fortran array (1:5, jsg:jeg, ksg:keg, 1:3) and inEijk
 * (1:6, jsg:jeg+1, ksg:keg+1, 1:3) as the coupler holds them (PsiSh = 5
 * shells), M0 the dipole moment of VecDipole (code units, m = (0, 0, M0)),
 * dtCpl the coupling time scale (code time), dtSW0 the nudging time scale
 * (the reference's one minute, 60 s / gT0). Needs the geometry and, with the
 * wind outside, gam_set_wind first (a wind time series is refused); call
 * before the initial condition, again whenever the coupler updates the
 * fields, and after every gam_set_wind. Also sets CalcDT's range to the
 * active cells (isDT..ieDT = is..ie, earthcmi.F90:136-142).
 * A tile of the magnetosphere away from the inner boundary (bc[0] =
 * GAM_BC_HALO) calls it too, with inExyz = inEijk = NULL: it takes the hooks
 * of its other sides (WindEFix and NudgeSW if its outer side is the wind,
 * FixEFieldLFM) and the DT range, as every rank of the reference's MPI run
 * does (EFix and PerStep test hasLowerBC / hasUpperBC). The k boundaries must
 * be periodic (the reference stops on a k decomposition of the magnetosphere,
 * earthcmi.F90:145-148). */
/* Ring averaging about the LFM axis (ring/doRing with ring/gid = "lfm":
 * InitRings ringutils.F90:37-236, RingAverage ringav.F90:26-75). A grid with
 * bc[2] and/or bc[3] = GAM_BC_LFM has the pole (the x axis) at js and/or
 * je+1; the other J side may be a tile's halo. The k boundaries must be
 * periodic with an even Nkp >= 8 (WrapK maps a ghost across the axis to
 * k + Nkp/2). Call before the geometry: the metric takes RingGridFix. With
 * it the step does what the reference does for such a grid:
 *   - the pole boundaries lfmIn / lfmOut (ghost cells take their conjugate
 *     across the axis, J and K face fluxes reversed) and RingFlux2FieldFix
 *     in every bFlux2Fld;
 *   - RingFlux (no flux through the pole faces) with FixGasFluxLFM, PoleE
 *     (with FixEFieldLFM) before the face update;
 *   - RingAverage after the update: the smoothing EMFs of the rings
 *     (Fourier modes 0..NFTmag of the ring fluxes removed, chunk averages
 *     reconstructed, modes put back), PoleE on them, E2Flux, CleanLoops
 *     (doClean, doFastClean), bFlux2Fld, SmoothGas (ring variables rho,
 *     momentum, internal energy chunk-averaged and reconstructed);
 *   - CalcDT after the ring average and the hooks (gamapp.F90:78-80);
 *   - with the ionosphere and the wind: the ring branches of IonInner,
 *     WindBC, WindEFix and NudgeSW.
 * NumR rings per pole with Nch[0..NumR-1] chunks each (each dividing Nkp;
 * gam_ring_defaults gives the reference's table by Nkp), recon the ring
 * reconstruction (ring/rngrec: 0 PPM, 1 PLM, 2 PCM), NFTmag the Fourier
 * modes removed from the fluxes (ringknobs/NMag, -1..2). The rings of the two
 * poles must not meet: Njp > 2 NumR + 2. The reference's defaults keep
 * doShift, doVClean and doMassRA off (and WENO reconstruction is not built).
 * The driver's own metric (gam_set_geometry_arrays) already holds
 * RingGridFix. */
int gam_set_rings(gam_handle* h, int32_t NumR, const int32_t* Nch, int32_t recon, int32_t NFTmag, int32_t doClean,
                  int32_t doFastClean);
/* The reference's default rings for Np cells around the axis (InitRings,
 * ringutils.F90:126-190; aggressive = ring/doAggressive): NumR and Nch[0..31].
 * GAM_EINVAL for an Np without defaults (the reference has none either). */
int gam_ring_defaults(int32_t Np, int32_t aggressive, int32_t* NumR, int32_t* Nch);

int gam_set_ionosphere(gam_handle* h, const double* inExyz, const double* inEijk, double M0, double dtCpl,
                       int32_t doIonPush, int32_t nIonP, double dtSW0);

/* ooState of the AB3 predictor (doAB3): its face fluxes (Fortran
 * magFlux(isg:ieg+1,...,1:3)) and time. The predictor reads nothing else of
 * ooState: the gas takes its third level from oState (mhdgroup.F90:500-502).
 * gam_upload_state with an oState sets ooState = oState at time otime - dt, the
 * fallback of readH5Restart for a restart without ooState (gioH5.F90:797-802);
 * a driver that holds ooState passes it here afterwards. The initial
 * conditions set ooState = State at time otime - dt (init.F90:232-241). */
int gam_set_oostate(gam_handle* h, const double* oomagFlux, double ootime);

/* Bounds-check build (libgamgpu_check.so, compiled with -DGAM_BOUNDS_CHECK):
 * every kernel checks the lowest and highest box index its stencils touch
 * before any load, and a failed check records the kernel (its position in the
 * step: 1 predictor, 2-7 Mom2Face/VxB, 8-10 fluxes, 11-12 update, 13 dt, 14
 * boundaries, 15 halo, 16 other) and the index, skips the access and makes
 * gam_step / gam_step_end / gam_calc_dt return GAM_EBOUNDS. Its device arrays
 * start filled with NaN (all bits set) instead of zeros, so a read of memory
 * nothing wrote shows up in the results. fired: 1 a check failed, 0 none,
 * -1 this library was built without the checks. */
int gam_bounds_status(gam_handle* h, int32_t* fired, int32_t* kernel, int64_t* index);
int gam_get_oostate(gam_handle* h, double* oomagFlux, double* ootime);

/* Dipole-in-wind start: the wind state in every active cell with the density
 * perturbed by amp*u (u uniform in [-1, 1), SplitMix64 of seed and the Fortran
 * cell index), the wind's uniform field as face fluxes of A = (B x r)/2
 * (VectorPot2Flux, gridutils.F90:193-237), then the initialisation order
 * above. Sets the wind boundary state when bc[1] = GAM_BC_WIND. Needs
 * gam_set_geometry, and the background field when doBackground. */
int gam_init_dipole_wind(gam_handle* h, const double wind[8], uint64_t seed, double amp);

/* Restart files: State and oState with ghosts, t, State/oState time, dt, dt0
 * and ts in one binary file (72-byte header "GAMRST01", then Gas, magFlux,
 * Bxyz, oGas, omagFlux as float64 Fortran-ordered arrays). Stands in for the
 * restart dump of writeH5Res / readH5Restart (src/gamera/gioH5.F90:636-858),
 * which is HDF5; reading needs a handle of the same grid size. */
int gam_write_restart(gam_handle* h, const char* path);
int gam_read_restart(gam_handle* h, const char* path);

/* Tiling (the MPI step of gamAppMpi_T, gamapp_mpi.F90:495-782): the grid cut
 * into tiles along i, j and k, one handle per tile (per GPU), with
 * GAM_BC_HALO on every side that faces a neighbour (both sides of a periodic
 * direction that is cut) and the grid's own boundary kinds on the others.
 * The functions named gam_halo_* / gam_set_slab_edges are the k-direction
 * forms kept for k-slabs (dir = 2). A step is
 *   gam_step_begin(h)                      predictor .. cell update
 *   gam_dt_partial(h, &bits, &nbad)        this slab's dt candidate
 *   (caller: min of bits and sum of nbad over all slabs, e.g. an NCCL
 *    all-reduce; bits are the IEEE-754 bits of a positive double, so the
 *    integer min is the double min)
 *   gam_step_end(h, bits, nbad, &dt, &t)   dt decision, local boundaries
 *   for dir = 0 (I), then 1 (J), then 2 (K), over the halo sides of dir:
 *     gam_tile_halo_pack(h, dir, 0|1, buf) / send / receive /
 *     gam_tile_halo_unpack(h, dir, 0|1, buf, 0)
 * Side 0 of a pack is what goes down to the tile below in dir (it fills that
 * tile's side-1 ghosts), side 1 what goes up. A pack covers the 4 layers next
 * to that side across the whole ghosted extent of the other two directions,
 * so exchanging the directions in turn, each after the previous one has been
 * unpacked on every tile, also fills the edge and corner ghosts. Buffers are
 * device memory of gam_tile_halo_bytes bytes; pack and unpack return after
 * their kernels finished. A pack or unpack of a side that is not a halo is
 * GAM_ESTATE. After a gam_init_*: exchange with copyB = 1 (Bxyz copied, like
 * the first EnforceBCs), then gam_init_finish_halo (oState = State, this
 * tile's CalcDT), min over tiles, gam_set_start(h, dt). Alternatively upload
 * a whole state with its ghosts (gam_upload_state). The tiles' states equal
 * the single grid's bit for bit, ghosts included. */
int gam_tile_halo_bytes(gam_handle* h, int32_t dir, int64_t* bytes);
int gam_tile_halo_pack(gam_handle* h, int32_t dir, int32_t side, void* dev_buf);
int gam_tile_halo_unpack(gam_handle* h, int32_t dir, int32_t side, const void* dev_buf, int32_t copyB);
/* Whether this tile is the lowest / highest in dir: CalcDT's range (isDT..ieDT
 * = is-1..ie+1, init.F90:511-530) takes the ghost layer below / above only on
 * the grid's own edges, not where a neighbour's cells are (and nowhere under
 * the magnetosphere's bounds). Call before the tile's gam_init_* (default:
 * both, as for the whole grid). */
int gam_set_tile_edges(gam_handle* h, int32_t dir, int32_t lowest, int32_t highest);
int gam_set_slab_edges(gam_handle* h, int32_t lowest, int32_t highest);
int gam_halo_bytes(gam_handle* h, int64_t* bytes);
int gam_halo_pack(gam_handle* h, int32_t side, void* dev_buf);
int gam_halo_unpack(gam_handle* h, int32_t side, const void* dev_buf, int32_t copyB);
int gam_init_finish_halo(gam_handle* h, double* dt_local);
int gam_set_start(gam_handle* h, double dt);
int gam_step_begin(gam_handle* h);
int gam_dt_partial(gam_handle* h, uint64_t* dtmin_bits, int32_t* nbad);
int gam_step_end(gam_handle* h, uint64_t dtmin_bits, int32_t nbad, double* dt, double* t);

/* The same tile step without host round trips, for a caller that reduces
 * on the device (an NCCL all-reduce of device buffers); the dt AllReduce(MIN)
 * of gamapp_mpi.F90:495-512 then never leaves the GPUs.
 *   gam_set_stream(h, stream)           enqueue all of this handle's work on
 *                                       the caller's stream (a non-default
 *                                       cudaStream_t; NULL: the handle's own);
 *                                       halo pack/unpack then return at once
 *   gam_step_begin_dev(h)               predictor .. cell update
 *   gam_dt_partial_dev(h, bits, nbad)   writes this slab's dt candidate bits
 *                                       and bad-cell count to the device
 *                                       int64 bits[0], nbad[0]
 *   (caller: MIN-reduce bits, SUM-reduce nbad over the slabs, in place)
 *   gam_step_end_dev(h, bits, nbad)     reads the reduced values from device
 *                                       memory: dt decision, local boundaries
 *   halo exchange as above
 *   gam_step_status(h, &dt, &t)         waits for the handle's stream; dt and
 *                                       t after the last step, and the status
 *                                       of the steps since the previous check
 * Every call only enqueues work (no host synchronisation) except
 * gam_step_status. A step that fails CalcDT halts the kernels of the later
 * steps and halo exchanges on the device (the state stays as the failing
 * step left it); every slab takes the same decision from the same reduced
 * values, and gam_step_status returns it (GAM_EDT_BAD / GAM_EDT_DISASTER).
 * No counterpart in the reference, whose MPI reduction is a host call. */
int gam_set_stream(gam_handle* h, void* stream);
int gam_step_begin_dev(gam_handle* h);
int gam_dt_partial_dev(gam_handle* h, int64_t* dtmin_bits, int64_t* nbad);
int gam_step_end_dev(gam_handle* h, const int64_t* dtmin_bits, const int64_t* nbad);
int gam_step_status(gam_handle* h, double* dt, double* t);

/* Flux stage of the step and its hand-written adjoint (differentiation form),
 * on caller-owned device arrays in the unpadded box layout: each field is
 * (nc, Nk+1, Nj+1, Ni+1) contiguous, i fastest, Ni = Nip + 8 (cell fields
 * leave the last slot of each axis unused). Inputs: QW = volume x half-state
 * primitives (5), Wn = limiter primitives (5), QB = volume x half-state Bxyz
 * (3), Blim = limiter Bxyz (3), Bnf = half-state flux / area (3), volume (1),
 * face (3), Tf (27: n + 9 d), fcB0 (9) and bFlux0 (3) in FP64 when
 * doBackground. gam_flux_forward writes gF (15: v + 5 d) and mF (9: x + 3 d)
 * over the face ranges of CalcStress (stress.F90:41-198); gam_flux_adjoint
 * adds the adjoints of those inputs for the given adjoints dgF, dmF (callers
 * zero dQW, dWn, dQB, dBlim, dBnf first). fp32 = 1: float arrays (fcB0/bFlux0
 * stay double). 8CENT reconstruction, 3-D; enqueued on stream (cudaStream_t,
 * 0 = default). No counterpart in the reference, which has no adjoint. */
int gam_flux_forward(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                     const void* Blim, const void* Bnf, const void* volume, const void* face, const void* Tf,
                     const double* fcB0, const double* bFlux0, void* gF, void* mF, void* stream);
int gam_flux_adjoint(const gam_params* p, int32_t fp32, const void* QW, const void* Wn, const void* QB,
                     const void* Blim, const void* Bnf, const void* volume, const void* face, const void* Tf,
                     const double* fcB0, const double* bFlux0, const void* dgF, const void* dmF, void* dQW,
                     void* dWn, void* dQB, void* dBlim, void* dBnf, void* stream);

/* Electric-field stage (CalcElecField: Mom2Face and the edge EMF loop,
 * fields.F90:70-517) and its hand-written adjoint, in the layout above.
 * Inputs: Dh = half-state density (1), abh = area x flux/max(area,TINY) (3),
 * bn = limiter flux/max(area,TINY) (3), VdV = volume x momentum/density (3),
 * volume, face (3), edge (3), Te (27), Teb (12), edgB0 (6, FP64) when
 * doBackground, dt; AVf is a 9-component scratch array. gam_efield_forward
 * writes E (3) over the edge ranges; gam_efield_adjoint adds the adjoints of
 * Dh, abh, bn and VdV for the adjoint dE (caller-zeroed outputs; dAVf is a
 * 3-component scratch array). No counterpart in the reference. */
int gam_efield_forward(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                       const void* VdV, const void* volume, const void* face, const void* edge, const void* Te,
                       const void* Teb, const double* edgB0, double dt, void* AVf, void* E, void* stream);
int gam_efield_adjoint(const gam_params* p, int32_t fp32, const void* Dh, const void* abh, const void* bn,
                       const void* VdV, const void* volume, const void* face, const void* edge, const void* Te,
                       const void* Teb, const double* edgB0, double dt, void* AVf, const void* dE, void* dDh,
                       void* dabh, void* dbn, void* dVdV, void* dAVf, void* stream);

/* Predictor (Predictor/PredictCell, mhdgroup.F90:444-615) and update
 * (applyUpdate/E2Flux/CellMaxwell, mhdgroup.F90:79-329, fields.F90:18-51)
 * stages and their hand-written adjoints, in the layout above; arrays are
 * passed as arrays of device pointers.
 * gam_predict_stage: st = {curGas, curMf, oldGas, oldMf}, geo = {volume, face,
 *   xfc, xyzcc, dxf (fp32 only: face centroid - cell centroid, 18)}, pdt = dt/2,
 *   odt = time - otime. Forward (out != NULL): out = {QW, Wn, Dh, VdV, QB, abh,
 *   Bnf, bn}. Adjoint (out == NULL): din = the adjoints of those eight, aB = a
 *   3-component scratch array; adds into dst = {dcurGas, dcurMf, doldGas,
 *   doldMf}. LFM limiter (doLFMLim = 1) only.
 * gam_update_stage: in = {curGas, curMf, E, gF, mF}, geo = {volume, xfc, xyzcc,
 *   dxf}, dpB0 (FP64) with doBackground. Forward: out = {nxtGas, nxtMf, nxtB
 *   (scratch)}. Adjoint: din = {dnxtGas, dnxtMf}, scratch sU (5) and sM (3);
 *   adds into dst = {dcurGas, dcurMf, dE, dgF, dmF}.
 * No counterpart in the reference. */
int gam_predict_stage(const gam_params* p, int32_t fp32, const void* const* st, const void* const* geo, double pdt,
                      double odt, void* const* out, const void* const* din, void* aB, void* const* dst, void* stream);
int gam_update_stage(const gam_params* p, int32_t fp32, const void* const* in, const void* const* geo,
                     const double* dpB0, double dt, void* const* out, const void* const* din, void* sU, void* sM,
                     void* const* dst, void* stream);

/* The non-periodic I boundaries of the differentiation form and their
 * adjoint, on caller-owned device arrays in the layout above (the step
 * restatement's boundary fills): bc[0] = GAM_BC_SPHIN (the SphIn copy of the
 * first active cell and its faces, bcs.F90:934-957) or GAM_BC_INFLOW (the
 * uniform inflow state and its face fluxes), bc[1] = GAM_BC_ZEROGRAD
 * (zeroGrad_obcI, bcs.F90:820-850) or GAM_BC_WIND (the constant solar wind
 * blended with the last active cell, apps/wind.F90:206-374, MinMach = 1),
 * on the 4 ghost layers of every (j, k); both I sides periodic is a no-op.
 * The tables are in the form's precision (FP64, or FP32 with fp32 = 1). */
typedef struct {
    double inflow[8];  /* bc[0] = GAM_BC_INFLOW: rho, P, Vx, Vy, Vz, Bx, By, Bz */
    double wind[8];    /* bc[1] = GAM_BC_WIND: the constant wind, same order */
    const void* wC;    /* bc[1] = GAM_BC_WIND: (Nk+8, Nj+8, 4) wind weight of ghost cell n of row (j, k) */
    const void* wF[3]; /* (Nk+9, Nj+9, 4): wind weight of the ghost faces of direction d */
    const void* sF[3]; /* (Nk+9, Nj+9, 4): the wind's flux through those faces */
} gam_iside;
/* gam_iside_fill fills the ghosts of Gas and mf in place; B = bFlux2Fld of
 * mf before the fill (zeroGrad_obcI and the wind read the last active cell's
 * field); geo = {face, Tf}. gam_iside_adjoint takes Gas and B as the fill
 * found them (it reads only the first and last active cells, which the fill
 * does not change) and the adjoints dGas, dMf of the filled arrays: in place,
 * every filled ghost passes its adjoint on and is zeroed; it adds into dB (the
 * adjoint of B) and, with bc[0] = GAM_BC_INFLOW and dinflow not NULL, into
 * the 8 adjoints of the inflow state (a device array, fixed-order sums).
 * No counterpart in the reference, which has no adjoint. */
int gam_iside_fill(const gam_params* p, int32_t fp32, const void* const* geo, const gam_iside* is, const void* B,
                   void* Gas, void* mf, void* stream);
int gam_iside_adjoint(const gam_params* p, int32_t fp32, const void* const* geo, const gam_iside* is,
                      const void* Gas, const void* B, void* dGas, void* dMf, void* dB, void* dinflow, void* stream);

/* One whole stepGamera of the differentiation form (fixed dt, AB2, 8CENT, no
 * Boris) and its adjoint, on caller-owned device arrays in the layout above:
 * the stages above plus the step's boundary conditions (periodic I and K,
 * periodic or zero-gradient J; bcs.F90:279-450, 853-892, applied in
 * EnforceBCs' order, step.F90:17-55) and bFlux2Fld (gridutils.F90:281-301);
 * the _iside variants below add the non-periodic I boundaries.
 * geo = {volume, face, xfc, xyzcc, dxf (fp32 only, else NULL), edge, Te, Teb,
 * Tf}; bg = {fcB0, bFlux0, edgB0, dpB0} (FP64) with doBackground, else NULL;
 * st = {curGas, curMf, oldGas, oldMf} (State and oState; the State's Bxyz is
 * bFlux2Fld of its fluxes, as EnforceBCs leaves it); dt and odt = time - otime
 * as for gam_predict_stage; work = gam_step_work_bytes bytes of device memory.
 * gam_step_fwd_save writes nxt = {nxtGas, nxtMf, nxtB} (the State after the
 * step, ghosts filled, Bxyz on every cell) and keeps the step's intermediate
 * arrays in work. gam_step_adj adds into dst = {dcurGas, dcurMf, doldGas,
 * doldMf} the adjoints of st for the adjoints dnxt = {dGas, dMf, dB} of nxt
 * (dB may be NULL); saved = 1 reuses the intermediates that gam_step_fwd_save
 * left in work for the same st, saved = 0 recomputes them first. The adjoint
 * sums every stencil's contributions in a fixed order (no atomics), so equal
 * inputs give equal bits on every call. Enqueued on stream (the adjoint forks
 * independent stages onto the library's own side streams of the device and
 * joins them back before it returns, so the work stays ordered on stream and
 * may be captured into a CUDA graph from it, once the first gam_step_adj call
 * on the same grid configuration and device has uploaded the tables of its
 * boundary-gather adjoint with synchronous copies); the stage and whole-step calls
 * of this form share device-global scratch scalars, so issue them from one
 * host thread per device. GAM_EINVAL for other boundaries, Boris, AB3, 7UP
 * or 2.5-D.
 * No counterpart in the reference, which has no adjoint. */
int gam_step_work_bytes(const gam_params* p, int32_t fp32, int64_t* bytes);
int gam_step_fwd_save(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                      const void* const* st, double dt, double odt, void* const* nxt, void* work, void* stream);
int gam_step_adj(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                 const void* const* st, double dt, double odt, int32_t saved, const void* const* dnxt,
                 void* const* dst, void* work, void* stream);
/* The same with the non-periodic I boundaries of gam_iside_fill (bc[0] =
 * GAM_BC_SPHIN or GAM_BC_INFLOW with bc[1] = GAM_BC_ZEROGRAD or GAM_BC_WIND):
 * after applyUpdate the step forms bFlux2Fld of the updated fluxes, fills
 * the I ghosts from it, then runs the copying boundaries of J and K and the
 * closing bFlux2Fld; the adjoint runs those backwards with
 * gam_iside_adjoint and, with bc[0] = GAM_BC_INFLOW and dinflow not NULL,
 * adds the adjoints of the 8 inflow values into the device array dinflow.
 * gam_step_fwd_save and gam_step_adj return GAM_EINVAL for these boundaries.
 * No counterpart in the reference. */
int gam_step_fwd_save_iside(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                            const gam_iside* is, const void* const* st, double dt, double odt, void* const* nxt,
                            void* work, void* stream);
int gam_step_adj_iside(const gam_params* p, int32_t fp32, const void* const* geo, const double* const* bg,
                       const gam_iside* is, const void* const* st, double dt, double odt, int32_t saved,
                       const void* const* dnxt, void* const* dst, void* dinflow, void* work, void* stream);

/* Conserved totals for callers that cannot allocate device memory.
 * No counterpart in the reference. Some callers cannot call cudaMalloc while
 * they run: their device memory belongs to another framework's pool, or they
 * reserve everything at start-up because allocation synchronises the device
 * and can fail once memory is fragmented. This entry point allocates nothing:
 * it reads the caller's device arrays State%Gas (Fortran layout, ghosts
 * included) and Grid%volume (cell-sized), enqueues the reduction on `stream`
 * (a cudaStream_t; 0 = default stream) and writes the five volume-weighted
 * totals (mass, momentum x/y/z, energy) to the caller's device buffer out[5].
 * Its block partial sums live in a fixed file-scope device array of 320 KiB,
 * held on every device that loads the library until the process exits, which
 * limits a call to Nip*Njp*Nkp <= 67,108,864 active cells; larger grids are
 * rejected with GAM_EINVAL and a message in err (errlen bytes, may be NULL).
 * The first call on a device looks up that array's address (set-up): make it
 * before any stream capture. The address is kept per device and context, and
 * looked up again when the device's context changes (after cudaDeviceReset).
 * Every call on a device shares that device's array and finds it holding the
 * last call's partial sums: calls whose kernels overlap on the same device
 * (for example enqueued on different streams) race; calls on different devices
 * do not, each device holding its own copy. An error left pending by an
 * earlier launch on the calling thread is returned as this call's GAM_ECUDA. */
int gam_totals_noalloc(const double* Gas, const double* volume, int32_t Nip, int32_t Njp, int32_t Nkp, double* out,
                       void* stream, char* err, int32_t errlen);

#ifdef __cplusplus
}
#endif
#endif /* GAMGPU_H */
