/*
 * windfvm.h - C ABI of the B200 (sm_100a) urban-wind FVM solver.
 *
 * This library is a drop-in for the HLSL compute-dispatch path of
 * puppy2333/UnityWindSimulation: the collocated, uniform-grid SIMPLE/PISO
 * time step with Smagorinsky LES and log-law wall functions that
 * FvmSolverController drives through IFvmSolver.Step().
 *
 *   reference interface             replaced by
 *   IFvmSolver (Assets/Code/FvmSolver/IFvmSolver.cs:3-24)
 *     FvmSolverGpu ctor (FvmSolverGpu.cs:173-222)        wf_create
 *     Step()            (FvmSolverGpu.cs:1050-1121)      wf_step
 *     InitFlags(int[])  (FvmSolverGpu.cs:972-987)        wf_init_flags
 *     InitVelPresFields (FvmSolverGpu.cs:790-896)        wf_init_vel_pres_fields
 *     SetFixedValueVelBndCond (FvmSolverGpu.cs:996-1022) wf_set_fixed_value_vel_bnd_cond
 *     ChangePhysFieldPos (FvmSolverGpu.cs:1026-1032)     wf_change_phys_field_pos
 *     ChangePhysDomainSize (FvmSolverGpu.cs:1034-1046)   (re-create the handle; see below)
 *     GetVelField/GetPresField/GetFlagField (:1568-1582) wf_get_vel / wf_get_pres / wf_get_flags
 *     gridType CollNonUniform + InitMeshBuffers (:682-788) wf_set_face_positions
 *
 * Conventions
 *   - Axes follow the reference: x streamwise, y vertical (ground at y = 0),
 *     z spanwise.  Host arrays are flat, x fastest: index = z*nx*ny + y*nx + x
 *     (InitShaderColl.compute:353, BuildingVoxelizer.cs:392).
 *   - Every entry point returns an int status (WF_OK = 0).  Nothing throws or
 *     aborts across the ABI.  wf_last_error(h) gives a message for the last
 *     failure on a handle, wf_strerror(status) a generic one.
 *   - A handle is not thread-safe.  All work of a handle runs on its own CUDA
 *     stream; blocking host copies synchronise that stream only.  Distinct
 *     handles may be used from distinct threads.
 *   - The library owns all device memory.  Host buffers are owned by the
 *     caller and copied synchronously.
 *   - All arithmetic is FP32.
 */
#ifndef WINDFVM_H
#define WINDFVM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WF_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
    WF_OK = 0,
    WF_ERR_INVALID_ARG = 1,  /* bad pointer, size, enum value or config      */
    WF_ERR_CUDA = 2,         /* a CUDA runtime call failed                   */
    WF_ERR_OOM = 3,          /* device allocation failed                     */
    WF_ERR_NONFINITE = 4,    /* NaN/Inf found in the solution                */
    WF_ERR_TIMEOUT = 5,      /* a bounded device wait gave up                */
    WF_ERR_UNSUPPORTED = 6,  /* option not implemented for this build        */
    WF_NOT_FINISHED = 7,     /* reserved for a time-budgeted step; no entry  */
                             /* point returns it: every step completes (the  */
                             /* reference's 30 ms slicing, FvmSolverGpu.cs:  */
                             /* 1267-1275, is dropped)                       */
    WF_ERR_STATE = 8,        /* call not valid in the handle's current state */
    WF_ERR_IO = 9            /* a file could not be created or written       */
};

/* ---- enums mirroring Constants.hlsl:4-14 and FluidSimConfig.cs:16-96 ---- */
enum { WF_CELL_FLUID = 0, WF_CELL_SOLID = 1 };
enum { WF_BND_FIXED_VALUE = 0, WF_BND_ZERO_GRAD = 1, WF_BND_SYMMETRY = 2 };
enum { WF_FACE_X0 = 0, WF_FACE_XN = 1, WF_FACE_Y0 = 2, WF_FACE_YN = 3,
       WF_FACE_Z0 = 4, WF_FACE_ZN = 5 };
enum { WF_SOLVER_SIMPLE = 0, WF_SOLVER_PISO = 1 };
enum { WF_TURB_NONE = 0, WF_TURB_SMAGORINSKY = 1 };
enum { WF_INFLOW_CONSTANT = 0, WF_INFLOW_LOG = 1 };

/* ---- reference-quirk switches (wf_config.compat_flags) ------------------
 * WF_COMPAT_RFLOAT_FACE_EDDY_VIS: faceEddyVisField is allocated RFloat
 *   (FvmSolverGpu.cs:304) but written/read as float4 (WallFunc.compute:189,
 *   FvmColl.compute:93).  Under D3D typed-UAV rules only .x survives, so the
 *   y- and z-normal wall viscosities read back as 0.  Set this flag to get the
 *   as-shipped behaviour; clear it (default) for the intended three channels.
 * WF_COMPAT_INIT_PROFILE_CELL_CENTRE: the reference initialises the interior
 *   log profile at y = j*dx (InitShaderColl.compute:120) but the inlet at
 *   (j+0.5)*dx (:279).  Set this flag to use (j+0.5)*dx for both.
 * WF_COMPAT_PISO_CONSISTENT: the reference PISO corrector uses nu only in
 *   A_od and no fixed-pressure boundary term (PisoColl.compute:135-169,
 *   200-253).  Set this flag to use nu + nu_t face viscosities and the
 *   fixed-pressure face term instead.  Default: reproduce the reference.     */
#define WF_COMPAT_RFLOAT_FACE_EDDY_VIS     0x1u
#define WF_COMPAT_INIT_PROFILE_CELL_CENTRE 0x2u
#define WF_COMPAT_PISO_CONSISTENT          0x4u

/* ---- configuration -------------------------------------------------------
 * Mirrors FluidSimConfig (FluidSimConfig.cs:113-178) + RuntimeConfig
 * (RuntimeConfig.cs:8-9) + the inflow constants hard-coded in
 * FvmSolverGpu.cs:816-819.  Fill it with wf_config_default() first.        */
typedef struct wf_config {
    uint32_t struct_size;       /* = sizeof(wf_config)                       */
    int32_t  nx, ny, nz;        /* gridRes (x streamwise, y vertical)        */
    float    dx;                /* cell size [m]; ds = dx^2, dv = dx^3       */
    float    dt;                /* time step [s]                             */
    float    mu;                /* dynamic viscosity; nu = mu / den          */
    float    den;               /* density                                   */
    float    ext_force[3];      /* externalForce                             */
    int32_t  vel_bc[6];         /* WF_BND_*, indexed by WF_FACE_*            */
    int32_t  pres_bc[6];        /* WF_BND_*, indexed by WF_FACE_*            */
    int32_t  solver_type;       /* WF_SOLVER_SIMPLE / WF_SOLVER_PISO         */
    int32_t  piso_correctors;   /* PISONumCorrectors                         */
    int32_t  turbulence;        /* WF_TURB_NONE / WF_TURB_SMAGORINSKY        */
    float    cs;                /* smagorinskyConstant                       */
    int32_t  vel_iters;         /* velMaxNumIter (Jacobi sweeps, momentum)   */
    int32_t  pres_iters;        /* presMaxNumIter (Jacobi sweeps, pressure)  */
    int32_t  inflow_type;       /* WF_INFLOW_CONSTANT / WF_INFLOW_LOG        */
    float    wind_speed;        /* RuntimeConfig.windSpeed (= velX0.x)       */
    float    inflow_ustar;      /* > 0: friction velocity used directly      */
    float    inflow_z0;         /* roughParam (reference: 1.0)               */
    float    inflow_kappa;      /* karmanConst (reference: 0.4)              */
    float    inflow_href;       /* refHeight (reference: 10.0)               */
    float    vel_zn[3];         /* velZn, fixed value on the Zn face         */
    int32_t  calc_residual;     /* calResidual                               */
    int32_t  vel_res_interval;  /* velResidualCheckInterval                  */
    int32_t  pres_res_interval; /* presResidualCheckInterval                 */
    float    vel_tol;           /* velTolerance                              */
    float    pres_tol;          /* presTolerance                             */
    uint32_t compat_flags;      /* WF_COMPAT_*                               */
    int32_t  check_finite;      /* != 0: wf_step returns WF_ERR_NONFINITE
                                   when the new fields hold NaN/Inf          */
    int32_t  use_graph;         /* != 0 (default): replay the step as a CUDA
                                   graph when the handle is in steady state  */
} wf_config;

/* Fills *cfg with the reference's FluidSimConfig defaults
 * (FluidSimConfig.cs:113-178) and the canonical urban boundary set of
 * Assets/Code/Config/AijBuilding0.asset (log inlet X0, zero-gradient/p=0
 * outlet Xn, wall Y0, symmetry Yn/Z0/Zn). */
void wf_config_default(wf_config* cfg);

/* ---- handle lifecycle ---------------------------------------------------- */
typedef struct wf_solver wf_solver;

/* Allocates every field and runs the constructor's set-up sequence
 * (FvmSolverGpu.cs:173-222): all cells fluid, initial fields, face eddy
 * viscosity 0, boundary planes.  SolidType.Box is not honoured: obstacles
 * come only through wf_init_flags.  `device` is a CUDA ordinal. */
int wf_create(const wf_config* cfg, int device, wf_solver** out);
int wf_destroy(wf_solver* h);

/* ---- IFvmSolver operations ----------------------------------------------- */
/* InitFlags(int[]): flags[i] > 0.5 marks cell i solid and zeroes its three
 * velocity buffers; otherwise the cell becomes fluid (CSInitModelFlag,
 * InitShaderColl.compute:346-364).  n = nx*ny*nz int32 values. */
int wf_init_flags(wf_solver* h, const int32_t* flags, size_t n);
/* InitVelPresFields(): constant or log-law interior velocity, p = 0
 * (CSInitVelPresFields / CSInitLogVelPresFields, InitShaderColl.compute:95-132). */
int wf_init_vel_pres_fields(wf_solver* h);
/* SetFixedValueVelBndCond() with RuntimeConfig.windSpeed = wind_speed
 * (CSSetFixedValueVelBndCond / CSSetLogVelBndCond, InitShaderColl.compute:253-285). */
int wf_set_fixed_value_vel_bnd_cond(wf_solver* h, float wind_speed);
/* ChangePhysFieldPos(): re-initialise the fields (FvmSolverGpu.cs:1026-1032). */
int wf_change_phys_field_pos(wf_solver* h);
/* Non-uniform collocated grid (FluidSimConfig.gridType = CollNonUniform,
 * FvmSolverGpu.cs:185-205; mesh buffers facePosX/Y/Z of InitMeshBuffers,
 * :682-788).  face_x[nx+1], face_y[ny+1], face_z[nz+1]: strictly increasing
 * face positions (cell x spans face_x[x]..face_x[x+1]).  From the next call
 * on, the step runs FvmCollNonUniform.compute's kernels (momentum and
 * pressure pre-computes, Jacobi sweeps, velocity correction), and
 * wf_init_vel_pres_fields / wf_set_fixed_value_vel_bnd_cond place a log
 * profile at the cells' centre heights (CSInitLogVelPresFieldsNonUniform,
 * CSSetLogVelBndCondNonUniform, InitShaderColl.compute:134-154,287-300);
 * call them after this, as the reference's constructor builds the mesh
 * before the fields.  The face-flux texture starts at zero and is bound
 * for the momentum kernels, which the reference leaves out (:1160,1196
 * are commented out).  SIMPLE, with or without the Smagorinsky model
 * (the wall function and LES kernels use the constant dx, as the
 * reference's WallFunc and Les shaders do; the momentum kernels interpolate
 * the eddy viscosity to the faces, useLES); PISO returns WF_ERR_UNSUPPORTED,
 * as the reference has no PISO shader for this grid (:493-496 throws);
 * batches and the adjoint take uniform grids only.  All three NULL: back to
 * the uniform grid. */
int wf_set_face_positions(wf_solver* h, const float* face_x, const float* face_y, const float* face_z);
/* The face-flux texture of the non-uniform grid (velFaceFluxField,
 * FvmSolverGpu.cs:275, written by CSPresCorrectRhieChowPreCompute,
 * FvmCollNonUniform.compute:1335-1341): three planes (x, y, z components)
 * of (nx+1)*(ny+1)*(nz+1) texels, x fastest. */
int wf_get_face_flux(wf_solver* h, float* out);
/* Writes the face-flux texture (same layout).  With wf_get_state /
 * wf_set_state it makes a checkpoint of a non-uniform handle exact: the
 * next step's momentum pre-compute reads the fluxes of the previous step. */
int wf_set_face_flux(wf_solver* h, const float* in);
/* InitVelPresFieldsFromBackGroundFlow (FvmSolverGpu.cs:898-929, kernel
 * CSInitVelPresFieldsFromBGFlowRotate, InitShaderColl.compute:185-226): sets
 * every cell's velocity (all iterate buffers) and pressure to the
 * background handle's current fields sampled trilinearly (clamped) at the
 * cell's position; corrections are zeroed.  pos / pos_bg: physical positions
 * of the two domains' centres (FluidSimConfig.physFieldPos), rot_deg: this
 * domain's rotation about the vertical axis (RuntimeConfig.
 * flowFieldOrientation).  As in the reference, a cell sits at (index -
 * res/2) * dx and the sampled vector is not rotated.  bg must be another
 * handle on the same device; it is not modified. */
int wf_init_from_background(wf_solver* h, const wf_solver* bg, const float pos[3], const float pos_bg[3],
                            float rot_deg);
/* Replaces the X0 inlet plane with caller data: ny*nz*3 floats, index
 * (z*ny + y)*3 + c (perturbed inflow).  The data are copied before the call
 * returns (through a page-locked staging buffer the handle allocates on
 * first use); the upload is ordered before the next step and does not wait
 * for the GPU. */
int wf_set_inflow_plane(wf_solver* h, const float* x0_plane_xyz);
/* Step() repeated n_steps times, each a complete time step with fixed
 * iteration counts (no 30 ms time slicing).  *ready (may be NULL) = 1. */
int wf_step(wf_solver* h, int n_steps, int* ready);
/* The steps of wf_step enqueued on the handle's stream without waiting for
 * them, as Unity's Dispatch calls return before the GPU runs them
 * (FvmSolverGpu.cs:1050-1121): a host can prepare the next inputs while the
 * GPU steps.  No finiteness check and no wf_last_step_ms update.  Every
 * call that reads fields to the host, wf_readback_wait and wf_sync wait for
 * the steps; a device fault surfaces at the next waiting call. */
int wf_step_async(wf_solver* h, int n_steps);
/* Waits for all work enqueued on the handle's stream. */
int wf_sync(wf_solver* h);
/* No counterpart in the reference.  The step rotates its buffers, so its
 * CUDA graph depends on which buffer holds which field; the few such states
 * repeat with a short period, and wf_step captures the graph of each state
 * the first time it meets it.  This call captures them all at once, without
 * running any step or changing any field, so that later wf_step calls only
 * replay.  Needs the replay state (use_graph on, calc_residual off, at least
 * one wf_step since the last field write); otherwise it does nothing. */
int wf_prepare_graphs(wf_solver* h);

/* ---- field access -------------------------------------------------------- */
enum { WF_LAYOUT_SOA = 0,   /* 3 planes of N floats: [c][z][y][x]           */
       WF_LAYOUT_XYZW = 1,  /* N float4 (x,y,z,0), the RenderTexture layout */
       WF_LAYOUT_XYZ = 2 }; /* N float3 interleaved                         */

/* Current velocity (velFieldLastTime after a step).  GetVelField (:1568-1571)
 * returns velFieldTex, which after the end-of-step swap (:1105) holds the
 * previous time level; wf_get_field(WF_FIELD_VEL) returns that texture. */
int wf_get_vel(wf_solver* h, float* out, int layout);
/* Current pressure (presFieldLastTime). N floats. */
int wf_get_pres(wf_solver* h, float* out);
/* Flag field, N int32 (0 fluid, 1 solid). */
int wf_get_flags(wf_solver* h, int32_t* out);
/* Velocity, pressure and step counter for an exact resume. vel: 3N floats
 * (SoA), pres: N floats. */
int wf_get_state(wf_solver* h, float* vel, float* pres, int64_t* step);

/* Asynchronous readback of the current velocity and pressure, for hosts that
 * read the fields every step (no counterpart on IFvmSolver; the reference's
 * exporter reads back the same way with AsyncGPUReadback,
 * NcFlowFieldExporter.cs:300-340).  wf_readback_begin snapshots the fields
 * on the solver's stream and copies them to the host buffers (vel in the
 * given layout, 3N or 4N floats; pres N floats) on a separate stream, so the
 * copy overlaps the following wf_step calls.  The buffers are complete after
 * wf_readback_wait; a second begin waits for the first.  Use page-locked host
 * memory (cudaHostAlloc, or torch pin_memory) for the copies to run
 * asynchronously. */
int wf_readback_begin(wf_solver* h, float* vel, float* pres, int layout);
int wf_readback_wait(wf_solver* h);
int wf_set_state(wf_solver* h, const float* vel, const float* pres, int64_t step);

/* Named fields of the reference's field set (MallocTextures,
 * FvmSolverGpu.cs:263-305) for per-kernel parity checks. */
enum {
    WF_FIELD_VEL = 0,                  /* velField            (vector) */
    WF_FIELD_VEL_LAST_TIME = 1,        /* velFieldLastTime    (vector) */
    WF_FIELD_VEL_LAST_ITER = 2,        /* velFieldLastIter    (vector) */
    WF_FIELD_VEL_CORRECT = 3,          /* velCorrectField     (vector) */
    WF_FIELD_PRES = 4,                 /* presFieldLastTime   (scalar) */
    WF_FIELD_PRES_CORRECT = 5,         /* presCorrectField    (scalar) */
    WF_FIELD_PRES_CORRECT_LAST_ITER = 6,/* presCorrectFieldLastIter    */
    WF_FIELD_D = 7,                    /* DField              (vector) */
    WF_FIELD_B = 8,                    /* bField              (vector) */
    WF_FIELD_DP = 9,                   /* DFieldPresCorrect   (scalar) */
    WF_FIELD_BP = 10,                  /* bFieldPresCorrect   (scalar) */
    WF_FIELD_AODU = 11,                /* AodUCorrectField    (vector) */
    WF_FIELD_EDDY_VIS = 12,            /* eddyVisField        (scalar) */
    WF_FIELD_FACE_EDDY_VIS = 13,       /* faceEddyVisField    (vector, W/S/D faces) */
    WF_FIELD_BND_X0 = 14,              /* boundary planes (vector):     */
    WF_FIELD_BND_XN = 15,              /*   X planes ny*nz, index z*ny+y */
    WF_FIELD_BND_Y0 = 16,              /*   Y planes nx*nz, index z*nx+x */
    WF_FIELD_BND_YN = 17,              /*   Z planes nx*ny, index y*nx+x */
    WF_FIELD_BND_Z0 = 18,
    WF_FIELD_BND_ZN = 19,
    WF_FIELD_DRAG = 20,                /* drag coefficient chi (scalar, 1/s); no
                                        * counterpart in the reference, see below */
    WF_FIELD_COUNT = 21
};
/* WF_FIELD_DRAG: Brinkman drag chi >= 0 per cell, added implicitly to the
 * momentum diagonal (D += dv * chi), which lets a soft (partly porous)
 * obstacle mask stand in for the binary flags, e.g. buildings whose heights
 * are continuous parameters.  Zero (the default, no storage) leaves the
 * reference's equations unchanged.  Setting it the first time drops the
 * handle's captured step graphs; rebuild batches that contain the handle. */
/* Number of cells (or plane points) of a field; vectors carry 3 floats per
 * point in SoA order. */
int wf_field_size(const wf_solver* h, int field, size_t* points, int* comps);
int wf_get_field(wf_solver* h, int field, float* out);
int wf_set_field(wf_solver* h, int field, const float* in);

/* Device pointers for zero-copy consumers (e.g. torch).  Valid until the
 * next wf_step / wf_step_async / wf_init_* / wf_set_* / wf_destroy.  Work
 * queued by wf_step_async may still be running: order reads after it on
 * `stream`, or call wf_sync first. */
typedef struct wf_device_fields {
    float*   vel[3];     /* velocity components (SoA planes), N floats each */
    float*   pres;       /* pressure, N floats                              */
    uint8_t* flags;      /* N bytes, 0 fluid / 1 solid                      */
    int64_t  n_cells;
    void*    stream;     /* the handle's cudaStream_t                       */
} wf_device_fields;
int wf_get_device_fields(wf_solver* h, wf_device_fields* out);

/* Residual norms of the last step, as the reference defines them
 * (FvmSolverGpu.cs:1232-1233,1361-1362): vel = sqrt(sum (D*du)^2 / 3N) of
 * the last momentum sweep, pres = sqrt(sum (Dp*dp')^2 / N) of the last
 * pressure sweep; mass = sum over fluid cells of |face-flux divergence| of
 * the final velocity.  Values are -1 when calc_residual was off. */
int wf_residuals(wf_solver* h, float* vel, float* pres, float* mass);
/* Mass imbalance sum |div u| (face-averaged fluxes, BC-aware) of the
 * current velocity; computed on demand. */
int wf_mass_imbalance(wf_solver* h, double* out);
/* Scans velocity and pressure for NaN/Inf: WF_OK or WF_ERR_NONFINITE. */
int wf_check_finite(wf_solver* h);

/* ---- per-kernel operations (parity checks against the CPU oracle) ------- */
/* Each runs exactly one reference kernel (or loop) on the handle's current
 * fields, with the reference's buffer roles and swaps. */
int wf_op_wallfunc(wf_solver* h);        /* CSCalLogLawWallFunc  WallFunc.compute:128-190 */
int wf_op_eddy_vis(wf_solver* h);        /* CSCalEddyVis         LES.compute:268-324      */
int wf_op_les_term(wf_solver* h);        /* CSCalLesDeferCorrectTerm LES.compute:327-687  */
int wf_op_vel_precompute(wf_solver* h);  /* CSVelPredictPreCompute FvmColl.compute:1292-1859 */
/* n sweeps of CSVelPredict (FvmColl.compute:1863-2069) with the swap of
 * FvmSolverGpu.cs:1265 after each and the final swap of :1279. */
int wf_op_vel_sweeps(wf_solver* h, int n);
int wf_op_pres_precompute(wf_solver* h); /* CSPresCorrectRhieChowPreCompute FvmColl.compute:2481-2787 */
/* n sweeps of CSPresCorrectRhieChow (FvmColl.compute:2790-2848), swaps as in
 * FvmSolverGpu.cs:1401,1415. */
int wf_op_pres_sweeps(wf_solver* h, int n);
int wf_op_apply_pres(wf_solver* h);      /* CSApplyPresCorrection FvmColl.compute:2851-2862 */
int wf_op_normalize(wf_solver* h);       /* CSPresNormalization  FvmColl.compute:2865-2880 (reference value read first) */
int wf_op_apply_vel(wf_solver* h);       /* CSApplyVelCorrectionDivergenceTheorem FvmColl.compute:2951-3121 */
int wf_op_zero_pres_correct(wf_solver* h); /* SetPresCorrectFieldtoZero FvmSolverGpu.cs:1545-1554 */
/* One PisoCorrection() (FvmSolverGpu.cs:1482-1533) with n pressure sweeps. */
int wf_op_piso(wf_solver* h, int n);
/* End of step: swap(velLastTime, vel); velLastIter <- velLastTime
 * (FvmSolverGpu.cs:1103-1118). */
int wf_op_end_step(wf_solver* h);
/* Residual kernels (FvmColl.compute:3124-3199) on the current fields. */
int wf_op_vel_residual(wf_solver* h, float* out);
int wf_op_pres_residual(wf_solver* h, float* out);

/* ---- diagnostics --------------------------------------------------------- */
const char* wf_last_error(const wf_solver* h);
const char* wf_strerror(int status);
int wf_version(void);   /* WF_ABI_VERSION */

/* Device time of the kernels of the last wf_step call, in milliseconds,
 * measured with CUDA events on the handle's stream. */
int wf_last_step_ms(const wf_solver* h, float* ms);

/* Building footprints rasterised into an int32 flag array (nx*ny*nz, index
 * (z*ny + y)*nx + x, 1 = solid) on `device`: boxes[5*b .. 5*b+4] =
 * (x0, x1, z0, z1, h) in cells, rotated by angle_deg about the domain centre
 * in the x-z plane and tested at cell centres; columns within `margin` cells
 * of the x/z boundaries stay fluid; a column is solid up to min(round(h),
 * ny - 1) cells of the tallest box containing it.  The flag layout is the one
 * BuildingVoxelizer produces for InitFlags (BuildingVoxelizer.cs:355-413);
 * the rasterisation itself (boxes instead of Unity meshes) has no counterpart
 * in the reference.  Allocates and frees device memory for the call. */
int wf_rasterise_boxes(int nx, int ny, int nz, const double* boxes, int n_boxes, double angle_deg, int margin,
                       int device, int32_t* flags);

/* Number of kernels this library launched inside wf_step calls since the
 * handle was created (graph replays count every kernel node). */
int wf_kernel_launches(const wf_solver* h, int64_t* total);

/* One step like wf_step(h, 1, NULL), enqueued kernel by kernel (no graph
 * replay) with a CUDA event between its phases; phase_ms[WF_PHASE_COUNT]
 * receives the device time of each phase (0 for phases the configuration
 * skips).  The fields end as after wf_step.  Host NVTX ranges name the step
 * and its phases for a profiler.  Replaces the reference's per-Step
 * Stopwatch log (FvmSolverGpu.cs:168-170,1111-1114), which timed host
 * dispatch only. */
enum {
    WF_PHASE_LES = 0,         /* wall function, eddy viscosity, LES term      */
    WF_PHASE_VEL_PRE = 1,     /* momentum D, b                                */
    WF_PHASE_VEL_SWEEPS = 2,  /* momentum Jacobi loop (coefficients included) */
    WF_PHASE_PRES_PRE = 3,    /* pressure-correction Dp, bp                   */
    WF_PHASE_PRES_SWEEPS = 4, /* pressure Jacobi loop (coefficients included) */
    WF_PHASE_CORRECT = 5,     /* apply p', normalisation, velocity correction */
    WF_PHASE_PISO = 6,        /* PISO correctors                              */
    WF_PHASE_END = 7,         /* end-of-step rotation                         */
    WF_PHASE_COUNT = 8
};
int wf_step_phases(wf_solver* h, float* phase_ms);

/* Times `reps` launches of one hot kernel of the step on the handle's
 * current coefficients, with CUDA events on the handle's stream; when
 * flush_l2 != 0 a 256 MiB buffer is written before each launch so every
 * launch starts with a cold L2.  Outputs: mean device time per launch, the
 * algorithmic bytes of one launch (the reference kernel's compulsory bytes
 * per cell times the cells and sweeps one launch covers) and the Jacobi
 * sweeps one launch performs.  The solver state is not modified. */
enum { WF_KERNEL_PRES_SWEEP = 0, WF_KERNEL_VEL_SWEEP = 1 };
int wf_time_kernel(wf_solver* h, int kernel, int reps, int flush_l2, float* ms_per_launch,
                   double* alg_bytes_per_launch, int* sweeps_per_launch);

/* ---- batched form ---------------------------------------------------------
 * Several independent cases (uneven grids, wind directions, inflow speeds,
 * building layouts) stepped together.  No counterpart in the reference,
 * which runs one domain per solver object (a second, background domain in
 * FvmSolverController.cs:143-151 is stepped separately, :472-480).  Every
 * case's step graph becomes an independent branch of one CUDA graph, so one
 * launch advances all cases by one step and the cases fill each other's idle
 * SMs.  Results are identical to stepping each handle alone.  All handles
 * must live on one device, use use_graph = 1 and calc_residual = 0. */
typedef struct wf_batch wf_batch;
int wf_batch_create(wf_solver* const* solvers, int n, wf_batch** out);
int wf_batch_destroy(wf_batch* b);    /* the handles stay valid */
int wf_batch_step(wf_batch* b, int n_steps);
/* Device time of the last wf_batch_step call (CUDA events), milliseconds. */
int wf_batch_last_step_ms(const wf_batch* b, float* ms);
int wf_batch_kernel_launches(const wf_batch* b, int64_t* total);
const char* wf_batch_last_error(const wf_batch* b);
/* Cases are dealt round-robin onto `width` chains that run concurrently; the
 * cases of one chain run one after another inside the same launch.  0
 * (default) = every case its own chain; 1 = all cases in sequence (keeps
 * each case's working set in L2 while it runs).  Speed only. */
int wf_batch_set_width(wf_batch* b, int width);
/* Captures the batch graphs of every buffer-role state the cases cycle
 * through (see wf_prepare_graphs), without stepping.  Needs every case in
 * the replay state (one wf_batch_step after creating the batch or changing
 * its width); otherwise it does nothing. */
int wf_batch_prepare_graphs(wf_batch* b);
/* How a batched step runs (no counterpart in the reference).
 * WF_BATCH_GRAPHS (default): every case's step graph as one branch of a
 * parent graph, as above.
 * WF_BATCH_PERSISTENT: every case's step is recorded as five captured
 * segments (its once-per-step kernels) around its four Jacobi loops
 * (momentum, SIMPLE pressure, two PISO pressure loops); each loop of all
 * cases then runs as ONE persistent cooperative launch whose blocks walk a
 * work queue of (case, tile) items sweep by sweep (pressure: K-sweep passes),
 * with a grid-wide barrier between sweeps.  Results are identical to the
 * graph mode.  All cases must have the same step structure (solver type,
 * correctors, turbulence, iteration counts).  Speed only. */
enum { WF_BATCH_GRAPHS = 0, WF_BATCH_PERSISTENT = 1 };
int wf_batch_set_mode(wf_batch* b, int mode);
int wf_batch_get_mode(const wf_batch* b, int* mode);
/* Upper bound of one grid-barrier wait in the persistent mode (default 2000
 * ms).  A wait that runs out sets an error word; every block of the launch
 * then returns without further waits, later loops of the step return at
 * once, and wf_batch_step returns WF_ERR_TIMEOUT (the cases' fields are then
 * not valid).  Nothing in a correct run waits near this long. */
int wf_batch_set_barrier_timeout(wf_batch* b, double ms);
/* Self-test of that bounded barrier: one cooperative launch of `blocks`
 * blocks (<= the device's SM count) that meet at a barrier expecting blocks +
 * extra arrivals, with the given time limit.  *status = WF_OK when the
 * barrier released (extra == 0), WF_ERR_TIMEOUT when its wait ran out (extra
 * > 0: arrivals that never come).  No counterpart in the reference. */
int wf_grid_barrier_selftest(int device, int blocks, int extra, double timeout_ms, int* status);
/* Self-test of the bounded stage waits of the TMA-staged pressure sweep (the
 * four-sweep pass the handle's pressure loops use where nx % 4 == 0): one
 * pass over the handle's current pressure coefficients into its host-I/O
 * staging buffer (no solver field is written), with every wait limited to
 * timeout_ms.  short_stage != 0 makes each block's first stage expect 16
 * bytes more than its loads deliver, so that wait runs out: every block then
 * returns after its loads in flight have landed.  *status = WF_OK when the
 * pass completed, WF_ERR_TIMEOUT when a wait ran out; WF_ERR_UNSUPPORTED
 * where the TMA pass does not apply.  The handle stays usable either way.
 * No counterpart in the reference. */
int wf_stage_wait_selftest(wf_solver* h, int short_stage, double timeout_ms, int* status);

/* Temporal-blocking depths of the Jacobi loops: pressure sweeps per pass
 * (1..4) and momentum sweeps per pass (1..2).  Results do not depend on
 * them; speed does, per grid size (see the autotuner in the Python host
 * package).  Drops the handle's captured step graphs; rebuild batches that
 * contain the handle afterwards. */
int wf_set_blocking(wf_solver* h, int pres_k, int vel_k);
int wf_get_blocking(const wf_solver* h, int* pres_k, int* vel_k);
/* Tile shapes of the Jacobi kernels: rows of the pressure multi-sweep tile
 * (32: 32 x 32 tiles, one block per SM; 16: 32 x 16 tiles, two blocks per
 * SM, more tiles for small grids) and the block of the four-cell momentum
 * sweep (vel_bx * vel_by * vel_bz == 256 threads; default 32 x 4 x 2).
 * Results do not depend on them.  Drops the handle's captured step graphs.
 * No counterpart in the reference (its kernels are [numthreads(8,8,8)]). */
int wf_set_tiles(wf_solver* h, int pres_rows, int vel_bx, int vel_by, int vel_bz);
int wf_get_tiles(const wf_solver* h, int* pres_rows, int* vel_bx, int* vel_by, int* vel_bz);

/* ---- field export ---------------------------------------------------------
 * NcFlowFieldExporter (NcFlowFieldExporter.cs:197-393): velocity and
 * pressure frames appended to a netCDF file while the solver runs.  Same
 * layout as the reference's file: dimensions time (unlimited), velX, velY,
 * velZ, velVec (4), presX, presY, presZ; coordinate variables at cell
 * centres ((i + 0.5) * dx); global attributes gridLayoutType = "Collocated"
 * and dt; variables time[time], velField[time][velZ][velY][velX][velVec]
 * (channels u, v, w, 0) and presField[time][presZ][presY][presX], all
 * float.  Written without libnetcdf as netCDF classic with 64-bit offsets
 * (CDF-2), which every netCDF reader opens.
 *
 * wf_export_frame queues the solver's current fields (the state after the
 * last wf_step): a device kernel packs the record, one asynchronous copy
 * moves it to a pinned host slot, a writer thread writes it.  `ring` pinned
 * slots (1..16) bound the frames in flight; the call blocks only while all
 * of them are being written.  wf_export_close drains the queue, writes the
 * record count and closes the file.  The solver must outlive the exporter.
 * File errors surface as WF_ERR_IO on the next call (wf_export_last_error). */
typedef struct wf_exporter wf_exporter;
int wf_export_open(wf_solver* h, const char* path, int save_vel, int save_pres, int ring, wf_exporter** out);
int wf_export_frame(wf_exporter* e, float phys_time);
int wf_export_frames_written(wf_exporter* e, int64_t* n);
const char* wf_export_last_error(const wf_exporter* e);
int wf_export_close(wf_exporter* e);

/* ---- discrete adjoint ------------------------------------------------------
 * No counterpart in the reference, which computes no derivatives.  The
 * vector-Jacobian product of the fixed-iteration step (momentum predictor,
 * SIMPLE correction, PISO correctors) is the same composition of maps
 * reversed: every Jacobi sweep becomes a transposed sweep, the once-per-step
 * maps scatter their local derivatives.  The forward step is recomputed from
 * a stored state with every Jacobi iterate kept.
 *
 * Supported: turbulence = 0, calc_residual = 0, at least one fixed-pressure
 * domain face (no normalisation), compat flag WF_COMPAT_PISO_CONSISTENT off.
 * wf_adj_create returns WF_ERR_UNSUPPORTED otherwise.  The adjoint handle
 * keeps a reference to `h`; destroy it before the solver. */
typedef struct wf_adjoint wf_adjoint;
int wf_adj_create(wf_solver* h, wf_adjoint** out);
int wf_adj_destroy(wf_adjoint* a);
const char* wf_adj_last_error(const wf_adjoint* a);

/* One step from the solver's current state (velocity and pressure), cut
 * after `phases` parts: 1 = momentum predictor, 2 = + SIMPLE pressure
 * correction, 3 = + PISO correctors (the whole step).  The solver does not
 * advance.  All arrays are host memory in the SoA layout.
 * wf_adj_step_forward: the state after the cut (u_out 3N, p_out N).
 * wf_adj_step_vjp: given adjoints of that output (ubar_out 3N, pbar_out N),
 * the adjoints of the input state (ubar_in 3N, pbar_in N) and, when
 * non-NULL, of the six boundary-value planes (gbar_planes: 3 * plane points
 * each, planes in WF_FACE_* order, as wf_field_size reports them) and of
 * the drag field (dragbar, N; defined whether or not a drag field is set). */
int wf_adj_step_forward(wf_adjoint* a, int phases, float* u_out, float* p_out);
int wf_adj_step_vjp(wf_adjoint* a, int phases, const float* ubar_out, const float* pbar_out, float* ubar_in,
                    float* pbar_in, float* gbar_planes, float* dragbar);

/* Pedestrian-comfort objective: the mean over the last `window` steps of the
 * mean squared speed |u|^2 on the fluid cells of one horizontal patch
 * (x0 <= x < x1, z0 <= z < z1 at height index y), divided by the patch's full
 * cell count. */
typedef struct wf_objective {
    int32_t x0, x1, z0, z1, y;
    int32_t window;
} wf_objective;

/* Advances the solver n_steps steps from its current state, evaluates the
 * objective and its derivatives with respect to the log-inflow parameters
 * (inflow_ustar, inflow_z0; needs inflow_type = WF_INFLOW_LOG with
 * inflow_ustar > 0).  include_init != 0 also differentiates the initial
 * interior profile of wf_init_vel_pres_fields (the current state must be that
 * profile).  dJ_ddrag (nullable, N floats): derivative with respect to the
 * drag field (WF_FIELD_DRAG), from which a soft building mask's height
 * gradients follow by the chain rule.  Steps that are not taped in the
 * forward pass are checkpointed every `checkpoint_every` steps and
 * recomputed (see wf_adj_set_max_tapes).  ms_forward / ms_total
 * (nullable): device time of the forward pass and of the whole call.
 * Derivatives are summed with float atomics: repeated calls agree to
 * rounding, not bit for bit. */
/* Device memory of the gradient: one step tape takes about
 * (3 nV + (nP + 1)(nC + 1) + 45) floats per cell.  wf_adj_gradient keeps as
 * many step tapes as device memory holds (at most max_tapes, 0 = no cap, and
 * at most n_steps), leaving room for the checkpoints and 1 GB.  The last R
 * steps of the window (R = the tapes kept) are taped during the forward pass
 * and reversed without recomputation; the earlier steps are checkpointed
 * every checkpoint_every steps and each segment is recomputed into tapes and
 * reversed.  When a segment's tapes do not all fit, the segments are
 * shortened to the tapes that fit (more checkpoints; each step recomputed
 * once), or, with wf_adj_set_segment_policy(a, 0) or when the extra
 * checkpoints do not fit, the segment's states are stored and it is
 * reversed in sub-blocks (each step recomputed twice).  The tapes stay
 * allocated until wf_adj_destroy.  Results do not depend on the split. */
int wf_adj_set_max_tapes(wf_adjoint* a, int max_tapes);
/* shorten = 1 (default): shorter segments when a segment's tapes do not fit;
 * 0: keep checkpoint_every and reverse in sub-blocks.  No reference
 * counterpart (the reference has no differentiated form). */
int wf_adj_set_segment_policy(wf_adjoint* a, int shorten);
int wf_adj_gradient(wf_adjoint* a, const wf_objective* obj, int n_steps, int checkpoint_every, int include_init,
                    double* J, double* dJ_dustar, double* dJ_dz0, float* dJ_ddrag, float* ms_forward,
                    float* ms_total);

/* ---- allocation-free residual --------------------------------------------
 * No counterpart in the reference.  For callers that must not allocate
 * device memory: an engine or visualiser plugin whose GPU memory belongs to
 * the host application, a real-time loop that cannot afford cudaMalloc's
 * implicit device synchronisation, a process with a locked-down allocator.
 *
 * Computes the continuity residual sqrt(sum_i (Dp_i*(p'_i - p'last_i))^2 / n)
 * (the same norm wf_residuals reports for the pressure loop) of caller-owned
 * device arrays of n_cells floats; d_pc_last may be NULL (all-zero iterate).
 * `stream` is a cudaStream_t (NULL: the legacy default stream); the call
 * returns after that stream has finished the reduction, with the norm in
 * *out (host memory).
 *
 * Scratch: a fixed array of WF_NOALLOC_BLOCKS + 1 doubles (32 KiB + 8 B)
 * compiled into the library; every GPU that loads the library holds it
 * until the process exits.  The call makes no cudaMalloc/cudaFree or other
 * allocating call.  Every call shares that array and overwrites what the
 * previous call left there, so calls that overlap on the GPU (different
 * streams or threads) race and must be serialised by the caller.  Every
 * call looks up the array's device address in the CUDA context current on
 * the calling thread (an address is not cached across contexts, so a host
 * context or a cudaDeviceReset between calls is safe); the first call in a
 * context also loads the library's device code there, so make that first
 * call before any stream capture.
 * Returns WF_ERR_INVALID_ARG for NULL inputs or when n_cells is < 1 or larger
 * than WF_NOALLOC_MAX_CELLS, WF_ERR_CUDA when a CUDA call fails. */
#define WF_NOALLOC_BLOCKS 4096
#define WF_NOALLOC_MAX_CELLS (WF_NOALLOC_BLOCKS * 256 * 64) /* 67,108,864 */
int wf_pres_residual_noalloc(const float* d_dp, const float* d_pc, const float* d_pc_last, int64_t n_cells,
                             void* stream, float* out);

#ifdef __cplusplus
}
#endif
#endif /* WINDFVM_H */
