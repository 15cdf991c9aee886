// ref_driver.cpp - the reference's own hot-path kernels, run on the CPU
// (test infrastructure only).
//
// oracle/ref_kernels.py turns the reference's compute shaders (FvmColl,
// PisoColl, LES, WallFunc, Utils) into C++ under oracle/_ref/; this file
// includes each one in its own namespace over oracle/hlsl_shim.h, owns the
// textures, binds them the way FvmSolverGpu binds them before each Dispatch
// and replays FvmSolverGpu.Step (FvmSolverGpu.cs:1050-1121) dispatch by
// dispatch.  Nothing here restates the numerics: every cell update is the
// reference's own kernel text.  The result is a second oracle that pins the
// C++ restatement (windfvm_oracle.cpp) and, through it, the CUDA library.
//
// Dispatch semantics.  A Dispatch runs every thread of the padded 8x8x8 grid
// ((res+7)/8 groups per axis, FvmSolverGpu.cs:1129 and the like); threads
// outside the region leave through the kernels' own InRegion checks.  All
// kernels of the step except one write only their own cell and read other
// cells only from textures they do not write, so their result does not
// depend on thread order and they run in parallel over z.  The exception is
// CSPresNormalization (FvmColl.compute, "presFieldLastTime[id] -= refPres"),
// which reads the reference cell that one of its own threads rewrites; the
// GPU gives no order, and this driver runs the reference cell's thread last,
// so every cell sees the value from before the dispatch.
//
// Texture formats.  faceEddyVisFieldTex is created RFloat
// (FvmSolverGpu.cs:304) while the shaders declare it float4: a store keeps
// only the first channel and a load returns (r, 0, 0, 1).  With
// WF_COMPAT_RFLOAT_FACE_EDDY_VIS set the driver applies exactly that after
// the wall-function dispatch (the only kernel that writes the texture);
// otherwise all three channels are kept, the intended behaviour.  The face
// texture is gridRes+1 per axis in the reference but only its first gridRes
// cells are ever written (CSCalLogLawWallFunc stores at its own cell), so it
// is held at gridRes here and the extra layer reads 0 as the never-written
// texels do.
//
// Not replayed: the residual kernels and early exit (calResidual; they need
// group-shared reductions and a host readback), and the 30 ms time slicing of
// VelPredict/PresCorrect, which depends on the wall clock; wfr_create rejects
// calc_residual != 0.  The kernels' globals are namespace-scope, so one
// wfr_solver steps at a time in a process.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "hlsl_shim.h"
#include "../include/windfvm.h"

namespace ref_fvm {
using namespace hlsl;
#include "_ref/fvm.inc"
}  // namespace ref_fvm
namespace ref_fvmnu {
using namespace hlsl;
#include "_ref/fvmnu.inc"
}  // namespace ref_fvmnu
namespace ref_piso {
using namespace hlsl;
#include "_ref/piso.inc"
}  // namespace ref_piso
namespace ref_les {
using namespace hlsl;
#include "_ref/les.inc"
}  // namespace ref_les
namespace ref_wall {
using namespace hlsl;
#include "_ref/wall.inc"
}  // namespace ref_wall
namespace ref_utils {
using namespace hlsl;
#include "_ref/utils.inc"
}  // namespace ref_utils
namespace ref_init {
using namespace hlsl;
#include "_ref/init.inc"
}  // namespace ref_init

using hlsl::float4;
using hlsl::int3;
using hlsl::uint3;

struct wfr_solver {
    wf_config cfg{};
    int nx = 0, ny = 0, nz = 0;
    size_t n = 0;
    float dx = 0, ds = 0, dv = 0, nu = 0;
    float wind = 0;  // RuntimeConfig.windSpeed
    // Textures, named after the FvmSolverGpu members they stand for.  The
    // "swaps" of FvmSolverGpu are swaps of these pointers.
    std::vector<float4> store4[8];
    std::vector<float> store1[6];
    std::vector<float4> bnd[6];
    std::vector<int> flag;
    float4 *vel, *velLastTime, *velLastIter, *velCorrect, *aodu, *D, *b, *face;
    float *pres, *pc, *pcLastIter, *Dp, *bp, *eddy;
    // Non-uniform collocated grid (gridType CollNonUniform): face positions
    // (facePosX/Y/Z, nx+1 / ny+1 / nz+1 entries, FvmSolverGpu.cs:682-788)
    // and velFaceFluxFieldTex ((nx+1)(ny+1)(nz+1) float3, :275).
    bool nonuniform = false;
    std::vector<float> fpx, fpy, fpz;
    std::vector<hlsl::float3> flux;
};

namespace {

// Every thread of a Dispatch over `res` with 8x8x8 groups.
template <class K>
void dispatch(const int3& res, K kernel) {
    const int gx = (res.x + 7) / 8 * 8, gy = (res.y + 7) / 8 * 8, gz = (res.z + 7) / 8 * 8;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < gz; ++z)
        for (int y = 0; y < gy; ++y)
            for (int x = 0; x < gx; ++x) kernel(uint3((unsigned)x, (unsigned)y, (unsigned)z));
}

uint3 group_of(uint3 id) { return uint3(id.x / 8, id.y / 8, id.z / 8); }
uint3 lane_of(uint3 id) { return uint3(id.x % 8, id.y % 8, id.z % 8); }

// Uniforms as FvmSolverGpu sets them: InitFvmShader (FvmSolverGpu.cs:370-396),
// InitPisoShader (:499-506), InitLesShader (:529-547), InitWallFuncShader
// (:565-585), InitUtilsShader (:594-596).
void set_uniforms(const wfr_solver& s) {
    const wf_config& c = s.cfg;
    const int3 res(s.nx, s.ny, s.nz);
    {
        using namespace ref_fvm;
        gridRes = res;
        velRes = res;
        presRes = res;
        dt = c.dt;
        dx = s.dx;
        ds = s.ds;
        dv = s.dv;
        nu = s.nu;
        den = c.den;
        externalForce = hlsl::float3(c.ext_force[0], c.ext_force[1], c.ext_force[2]);
        numGroups = int3((s.nx + 7) / 8, (s.ny + 7) / 8, (s.nz + 7) / 8);
        useLES = c.turbulence == WF_TURB_SMAGORINSKY;
        velBndTypeX0 = c.vel_bc[WF_FACE_X0];
        velBndTypeXn = c.vel_bc[WF_FACE_XN];
        velBndTypeY0 = c.vel_bc[WF_FACE_Y0];
        velBndTypeYn = c.vel_bc[WF_FACE_YN];
        velBndTypeZ0 = c.vel_bc[WF_FACE_Z0];
        velBndTypeZn = c.vel_bc[WF_FACE_ZN];
        presBndTypeX0 = c.pres_bc[WF_FACE_X0];
        presBndTypeXn = c.pres_bc[WF_FACE_XN];
        presBndTypeY0 = c.pres_bc[WF_FACE_Y0];
        presBndTypeYn = c.pres_bc[WF_FACE_YN];
        presBndTypeZ0 = c.pres_bc[WF_FACE_Z0];
        presBndTypeZn = c.pres_bc[WF_FACE_ZN];
    }
    {
        // InitFvmNonUniformShader (FvmSolverGpu.cs:446-480): the same
        // uniforms without dx/ds/dv, which the kernels take from facePos.
        using namespace ref_fvmnu;
        gridRes = res;
        dt = c.dt;
        nu = s.nu;
        den = c.den;
        externalForce = hlsl::float3(c.ext_force[0], c.ext_force[1], c.ext_force[2]);
        numGroups = int3((s.nx + 7) / 8, (s.ny + 7) / 8, (s.nz + 7) / 8);
        useLES = c.turbulence == WF_TURB_SMAGORINSKY;
        velBndTypeX0 = c.vel_bc[WF_FACE_X0];
        velBndTypeXn = c.vel_bc[WF_FACE_XN];
        velBndTypeY0 = c.vel_bc[WF_FACE_Y0];
        velBndTypeYn = c.vel_bc[WF_FACE_YN];
        velBndTypeZ0 = c.vel_bc[WF_FACE_Z0];
        velBndTypeZn = c.vel_bc[WF_FACE_ZN];
        presBndTypeX0 = c.pres_bc[WF_FACE_X0];
        presBndTypeXn = c.pres_bc[WF_FACE_XN];
        presBndTypeY0 = c.pres_bc[WF_FACE_Y0];
        presBndTypeYn = c.pres_bc[WF_FACE_YN];
        presBndTypeZ0 = c.pres_bc[WF_FACE_Z0];
        presBndTypeZn = c.pres_bc[WF_FACE_ZN];
    }
    {
        using namespace ref_piso;
        gridRes = res;
        dt = c.dt;
        dx = s.dx;
        ds = s.ds;
        dv = s.dv;
        nu = s.nu;
        den = c.den;
        externalForce = hlsl::float3(c.ext_force[0], c.ext_force[1], c.ext_force[2]);
    }
    {
        using namespace ref_les;
        gridRes = res;
        dx = s.dx;
        ds = s.ds;
        nu = s.nu;
        cs = c.cs;
        velBndTypeX0 = c.vel_bc[WF_FACE_X0];
        velBndTypeXn = c.vel_bc[WF_FACE_XN];
        velBndTypeY0 = c.vel_bc[WF_FACE_Y0];
        velBndTypeYn = c.vel_bc[WF_FACE_YN];
        velBndTypeZ0 = c.vel_bc[WF_FACE_Z0];
        velBndTypeZn = c.vel_bc[WF_FACE_ZN];
        presBndTypeX0 = c.pres_bc[WF_FACE_X0];
        presBndTypeXn = c.pres_bc[WF_FACE_XN];
        presBndTypeY0 = c.pres_bc[WF_FACE_Y0];
        presBndTypeYn = c.pres_bc[WF_FACE_YN];
        presBndTypeZ0 = c.pres_bc[WF_FACE_Z0];
        presBndTypeZn = c.pres_bc[WF_FACE_ZN];
    }
    {
        using namespace ref_wall;
        gridRes = res;
        dx = s.dx;
        ds = s.ds;
        nu = s.nu;
        den = c.den;
        cs = c.cs;
        velBndTypeX0 = c.vel_bc[WF_FACE_X0];
        velBndTypeXn = c.vel_bc[WF_FACE_XN];
        velBndTypeY0 = c.vel_bc[WF_FACE_Y0];
        velBndTypeYn = c.vel_bc[WF_FACE_YN];
        velBndTypeZ0 = c.vel_bc[WF_FACE_Z0];
        velBndTypeZn = c.vel_bc[WF_FACE_ZN];
        presBndTypeX0 = c.pres_bc[WF_FACE_X0];
        presBndTypeXn = c.pres_bc[WF_FACE_XN];
        presBndTypeY0 = c.pres_bc[WF_FACE_Y0];
        presBndTypeYn = c.pres_bc[WF_FACE_YN];
        presBndTypeZ0 = c.pres_bc[WF_FACE_Z0];
        presBndTypeZn = c.pres_bc[WF_FACE_ZN];
    }
    {
        using namespace ref_utils;
        gridRes = res;
        velRes = res;
        presRes = res;
    }
    {
        // InitInitShader (:306-330), InitVelPresFields (:812-820) and
        // SetFixedValueVelBndCond (:1004-1010).  The reference hard-codes
        // karmanConst 0.4, roughParam 1 and refHeight 10; the config's
        // defaults are those values.
        using namespace ref_init;
        gridRes = res;
        velX0 = hlsl::float3(s.wind, 0.f, 0.f);
        velZn = hlsl::float3(c.vel_zn[0], c.vel_zn[1], c.vel_zn[2]);
        internalVelField = hlsl::float3(s.wind, 0.f, 0.f);
        dx = s.dx;
        karmanConst = c.inflow_kappa;
        roughParam = c.inflow_z0;
        refHeight = c.inflow_href;
    }
}

// SetBndTextures (FvmSolverGpu.cs:1556-1564) for one shader namespace.
template <class T2>
void bind_bnd(wfr_solver& s, T2& x0, T2& xn, T2& y0, T2& yn, T2& z0, T2& zn) {
    x0.bind(s.bnd[WF_FACE_X0].data(), s.ny, s.nz);
    xn.bind(s.bnd[WF_FACE_XN].data(), s.ny, s.nz);
    y0.bind(s.bnd[WF_FACE_Y0].data(), s.nx, s.nz);
    yn.bind(s.bnd[WF_FACE_YN].data(), s.nx, s.nz);
    z0.bind(s.bnd[WF_FACE_Z0].data(), s.nx, s.ny);
    zn.bind(s.bnd[WF_FACE_ZN].data(), s.nx, s.ny);
}

// Binds every texture of every shader to the driver's current roles.  The
// reference binds a subset per kernel; binding all of them to the same roles
// is equivalent, because a kernel only touches the textures it declares and
// the host binds each declared texture to this role before every Dispatch.
void bind_all(wfr_solver& s) {
    const int X = s.nx, Y = s.ny, Z = s.nz;
    {
        using namespace ref_fvm;
        velField.bind(s.vel, X, Y, Z);
        velFieldLastTime.bind(s.velLastTime, X, Y, Z);
        velFieldLastIter.bind(s.velLastIter, X, Y, Z);
        velCorrectField.bind(s.velCorrect, X, Y, Z);
        presFieldLastTime.bind(s.pres, X, Y, Z);
        presCorrectField.bind(s.pc, X, Y, Z);
        presCorrectFieldLastIter.bind(s.pcLastIter, X, Y, Z);
        flagField.bind(s.flag.data(), X, Y, Z);
        DField.bind(s.D, X, Y, Z);
        bField.bind(s.b, X, Y, Z);
        DFieldPresCorrect.bind(s.Dp, X, Y, Z);
        bFieldPresCorrect.bind(s.bp, X, Y, Z);
        AodUCorrectField.bind(s.aodu, X, Y, Z);
        eddyVisField.bind(s.eddy, X, Y, Z);
        faceEddyVisField.bind(s.face, X, Y, Z);
        bind_bnd(s, bndFieldX0, bndFieldXn, bndFieldY0, bndFieldYn, bndFieldZ0, bndFieldZn);
    }
    {
        // The non-uniform shader.  velFaceFluxField is bound for every
        // kernel here; see set_face_positions for the binding the reference
        // leaves out.
        using namespace ref_fvmnu;
        velField.bind(s.vel, X, Y, Z);
        velFieldLastTime.bind(s.velLastTime, X, Y, Z);
        velFieldLastIter.bind(s.velLastIter, X, Y, Z);
        velCorrectField.bind(s.velCorrect, X, Y, Z);
        presFieldLastTime.bind(s.pres, X, Y, Z);
        presCorrectField.bind(s.pc, X, Y, Z);
        presCorrectFieldLastIter.bind(s.pcLastIter, X, Y, Z);
        flagField.bind(s.flag.data(), X, Y, Z);
        DField.bind(s.D, X, Y, Z);
        bField.bind(s.b, X, Y, Z);
        DFieldPresCorrect.bind(s.Dp, X, Y, Z);
        bFieldPresCorrect.bind(s.bp, X, Y, Z);
        AodUCorrectField.bind(s.aodu, X, Y, Z);
        eddyVisField.bind(s.eddy, X, Y, Z);
        if (s.nonuniform) {
            velFaceFluxField.bind(s.flux.data(), X + 1, Y + 1, Z + 1);
            facePosX.p = s.fpx.data();
            facePosX.n = s.fpx.size();
            facePosY.p = s.fpy.data();
            facePosY.n = s.fpy.size();
            facePosZ.p = s.fpz.data();
            facePosZ.n = s.fpz.size();
        }
        bind_bnd(s, bndFieldX0, bndFieldXn, bndFieldY0, bndFieldYn, bndFieldZ0, bndFieldZn);
    }
    {
        using namespace ref_piso;
        velField.bind(s.vel, X, Y, Z);
        velFieldLastTime.bind(s.velLastTime, X, Y, Z);
        velFieldLastIter.bind(s.velLastIter, X, Y, Z);
        velCorrectField.bind(s.velCorrect, X, Y, Z);
        presFieldLastTime.bind(s.pres, X, Y, Z);
        presCorrectField.bind(s.pc, X, Y, Z);
        presCorrectFieldLastIter.bind(s.pcLastIter, X, Y, Z);
        flagField.bind(s.flag.data(), X, Y, Z);
        DField.bind(s.D, X, Y, Z);
        AodUCorrectField.bind(s.aodu, X, Y, Z);
    }
    {
        using namespace ref_les;
        velFieldLastTime.bind(s.velLastTime, X, Y, Z);
        flagField.bind(s.flag.data(), X, Y, Z);
        eddyVisField.bind(s.eddy, X, Y, Z);
        bField.bind(s.b, X, Y, Z);
        faceEddyVisField.bind(s.face, X, Y, Z);
        bind_bnd(s, bndFieldX0, bndFieldXn, bndFieldY0, bndFieldYn, bndFieldZ0, bndFieldZn);
    }
    {
        using namespace ref_wall;
        velFieldLastTime.bind(s.velLastTime, X, Y, Z);
        flagField.bind(s.flag.data(), X, Y, Z);
        faceEddyVisField.bind(s.face, X, Y, Z);
        bind_bnd(s, bndFieldX0, bndFieldXn, bndFieldY0, bndFieldYn, bndFieldZ0, bndFieldZn);
    }
}

int3 res_of(const wfr_solver& s) { return int3(s.nx, s.ny, s.nz); }

// ---- FvmSolverGpu stages --------------------------------------------------

void cal_wall_func(wfr_solver& s) {  // CalWallFunc, FvmSolverGpu.cs:1140-1147
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_wall::CSCalLogLawWallFunc(id); });
    if (s.cfg.compat_flags & WF_COMPAT_RFLOAT_FACE_EDDY_VIS)
        for (size_t i = 0; i < s.n; ++i) s.face[i] = float4(s.face[i].x, 0.f, 0.f, 1.f);
}

void cal_les_terms(wfr_solver& s) {  // CalLesTerms, :1123-1138
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_les::CSCalEddyVis(id); });
    dispatch(res_of(s), [](uint3 id) { ref_les::CSCalLesDeferCorrectTerm(id); });
}

void vel_predict(wfr_solver& s) {  // VelPredict, :1238-1282, without residual checks
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvm::CSVelPredictPreCompute(id); });
    for (int k = 0; k < s.cfg.vel_iters; ++k) {
        bind_all(s);
        dispatch(res_of(s), [](uint3 id) { ref_fvm::CSVelPredict(id); });
        std::swap(s.velLastIter, s.vel);
    }
    std::swap(s.velLastIter, s.vel);
}

bool has_fixed_pressure(const wf_config& c) {
    for (int f = 0; f < 6; ++f)
        if (c.pres_bc[f] == WF_BND_FIXED_VALUE) return true;
    return false;
}

void pres_correct(wfr_solver& s) {  // PresCorrect, :1367-1439, without residual checks
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvm::CSPresCorrectRhieChowPreCompute(id); });
    for (int k = 0; k < s.cfg.pres_iters; ++k) {
        bind_all(s);
        dispatch(res_of(s), [](uint3 id) { ref_fvm::CSPresCorrectRhieChow(id); });
        std::swap(s.pcLastIter, s.pc);
    }
    std::swap(s.pcLastIter, s.pc);
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvm::CSApplyPresCorrection(id); });
    if (!has_fixed_pressure(s.cfg)) {
        // CSPresNormalization with the reference cell's thread last (see the
        // file comment).  Serial: the kernel reads a cell it also writes.
        const uint3 ref_cell(2u, (unsigned)(s.ny / 2), 2u);
        const int gx = (s.nx + 7) / 8 * 8, gy = (s.ny + 7) / 8 * 8, gz = (s.nz + 7) / 8 * 8;
        for (int z = 0; z < gz; ++z)
            for (int y = 0; y < gy; ++y)
                for (int x = 0; x < gx; ++x) {
                    const uint3 id((unsigned)x, (unsigned)y, (unsigned)z);
                    if (id.x == ref_cell.x && id.y == ref_cell.y && id.z == ref_cell.z) continue;
                    ref_fvm::CSPresNormalization(id);
                }
        ref_fvm::CSPresNormalization(ref_cell);
    }
}

void apply_vel_correction(wfr_solver& s) {  // ApplyVelCorrection, :1441-1480 (collocated)
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvm::CSApplyVelCorrectionDivergenceTheorem(id); });
}

void set_pres_value(wfr_solver& s, float* dest, float value) {  // CSSetPresField
    ref_utils::presValue = value;
    ref_utils::destPres.bind(dest, s.nx, s.ny, s.nz);
    dispatch(res_of(s), [](uint3 id) { ref_utils::CSSetPresField(id); });
}

void set_pres_correct_to_zero(wfr_solver& s) {  // SetPresCorrectFieldtoZero, :1545-1554
    set_pres_value(s, s.pc, 0.f);
    set_pres_value(s, s.pcLastIter, 0.f);
}

void copy_vel_field(wfr_solver& s, float4* dest, float4* src) {  // CopyVelField, :1537-1543
    ref_utils::destVel.bind(dest, s.nx, s.ny, s.nz);
    ref_utils::srcVel.bind(src, s.nx, s.ny, s.nz);
    dispatch(res_of(s), [](uint3 id) { ref_utils::CSCopyVelField(id); });
}

void piso_correction(wfr_solver& s) {  // PisoCorrection, :1482-1535
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_piso::CSPisoCalAodUCorrect(id, group_of(id), lane_of(id)); });
    for (int k = 0; k < s.cfg.pres_iters; ++k) {
        bind_all(s);
        dispatch(res_of(s), [](uint3 id) { ref_piso::CSPisoPresCorrection(id, group_of(id), lane_of(id)); });
        std::swap(s.pcLastIter, s.pc);
    }
    std::swap(s.pcLastIter, s.pc);
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_piso::CSPisoApplyPresCorrection(id); });
    dispatch(res_of(s), [](uint3 id) { ref_piso::CSPisoVelCorrection(id, group_of(id), lane_of(id)); });
    set_pres_correct_to_zero(s);
}

// The same stages over the non-uniform shader (gridType CollNonUniform):
// _VelPredictPreCompute / _VelPredictCollAccelerated (:1149-1168,
// :1185-1203), _PresCorrectPreCompute / _PresCorrectCollAccelerated
// (:1284-1330), PresCorrect's apply and normalisation (:1367-1439) and
// ApplyVelCorrection (:1441-1480).  SIMPLE without turbulence only (see
// wfr_set_face_positions).
void vel_predict_nu(wfr_solver& s) {
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvmnu::CSVelPredictPreCompute(id); });
    for (int k = 0; k < s.cfg.vel_iters; ++k) {
        bind_all(s);
        dispatch(res_of(s), [](uint3 id) { ref_fvmnu::CSVelPredict(id); });
        std::swap(s.velLastIter, s.vel);
    }
    std::swap(s.velLastIter, s.vel);
}

void pres_correct_nu(wfr_solver& s) {
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvmnu::CSPresCorrectRhieChowPreCompute(id); });
    for (int k = 0; k < s.cfg.pres_iters; ++k) {
        bind_all(s);
        dispatch(res_of(s), [](uint3 id) { ref_fvmnu::CSPresCorrectRhieChow(id); });
        std::swap(s.pcLastIter, s.pc);
    }
    std::swap(s.pcLastIter, s.pc);
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvmnu::CSApplyPresCorrection(id); });
    if (!has_fixed_pressure(s.cfg)) {
        const uint3 ref_cell(2u, (unsigned)(s.ny / 2), 2u);
        const int gx = (s.nx + 7) / 8 * 8, gy = (s.ny + 7) / 8 * 8, gz = (s.nz + 7) / 8 * 8;
        for (int z = 0; z < gz; ++z)
            for (int y = 0; y < gy; ++y)
                for (int x = 0; x < gx; ++x) {
                    const uint3 id((unsigned)x, (unsigned)y, (unsigned)z);
                    if (id.x == ref_cell.x && id.y == ref_cell.y && id.z == ref_cell.z) continue;
                    ref_fvmnu::CSPresNormalization(id);
                }
        ref_fvmnu::CSPresNormalization(ref_cell);
    }
}

void step_once_nu(wfr_solver& s) {  // Step, :1050-1121, on the non-uniform grid
    set_uniforms(s);
    if (s.cfg.turbulence == WF_TURB_SMAGORINSKY) {  // the Les and WallFunc shaders, constant dx
        cal_wall_func(s);
        cal_les_terms(s);
    }
    vel_predict_nu(s);
    pres_correct_nu(s);
    bind_all(s);
    dispatch(res_of(s), [](uint3 id) { ref_fvmnu::CSApplyVelCorrectionDivergenceTheorem(id); });
    set_pres_correct_to_zero(s);
    std::swap(s.velLastTime, s.vel);
    copy_vel_field(s, s.velLastIter, s.velLastTime);
}

void step_once(wfr_solver& s) {  // Step, :1050-1121, every stage finishing in one call
    set_uniforms(s);
    if (s.cfg.turbulence == WF_TURB_SMAGORINSKY) {
        cal_wall_func(s);
        cal_les_terms(s);
    }
    vel_predict(s);
    pres_correct(s);
    apply_vel_correction(s);
    set_pres_correct_to_zero(s);
    if (s.cfg.solver_type == WF_SOLVER_PISO)
        for (int c = 0; c < s.cfg.piso_correctors; ++c) piso_correction(s);
    std::swap(s.velLastTime, s.vel);
    copy_vel_field(s, s.velLastIter, s.velLastTime);
}

// ---- set-up (InitShaderColl.compute) -------------------------------------

void bind_init(wfr_solver& s) {
    const int X = s.nx, Y = s.ny, Z = s.nz;
    using namespace ref_init;
    velField.bind(s.vel, X, Y, Z);
    velFieldLastTime.bind(s.velLastTime, X, Y, Z);
    velFieldLastIter.bind(s.velLastIter, X, Y, Z);
    velCorrectField.bind(s.velCorrect, X, Y, Z);
    presFieldLastTime.bind(s.pres, X, Y, Z);
    presCorrectField.bind(s.pc, X, Y, Z);
    presCorrectFieldLastIter.bind(s.pcLastIter, X, Y, Z);
    flagField.bind(s.flag.data(), X, Y, Z);
    faceEddyVisField.bind(s.face, X, Y, Z);
    bind_bnd(s, bndFieldX0, bndFieldXn, bndFieldY0, bndFieldYn, bndFieldZ0, bndFieldZn);
    facePosX.p = s.nonuniform ? s.fpx.data() : nullptr;
    facePosX.n = s.fpx.size();
    facePosY.p = s.nonuniform ? s.fpy.data() : nullptr;
    facePosY.n = s.fpy.size();
    facePosZ.p = s.nonuniform ? s.fpz.data() : nullptr;
    facePosZ.n = s.fpz.size();
}

// InitVelPresFields, :786-860; on the non-uniform grid the log profile is
// CSInitLogVelPresFieldsNonUniform (:835-876, kernel looked up at :329-332).
void init_vel_pres_fields(wfr_solver& s) {
    set_uniforms(s);
    bind_init(s);
    if (s.cfg.inflow_type == WF_INFLOW_LOG && s.nonuniform)
        dispatch(res_of(s), [](uint3 id) { ref_init::CSInitLogVelPresFieldsNonUniform(id); });
    else if (s.cfg.inflow_type == WF_INFLOW_LOG)
        dispatch(res_of(s), [](uint3 id) { ref_init::CSInitLogVelPresFields(id); });
    else
        dispatch(res_of(s), [](uint3 id) { ref_init::CSInitVelPresFields(id); });
}

// SetFixedValueVelBndCond, :998-1022 (CSSetLogVelBndCondNonUniform on the
// non-uniform grid, :338-341).
void set_fixed_value_vel_bnd_cond(wfr_solver& s) {
    set_uniforms(s);
    bind_init(s);
    if (s.cfg.inflow_type == WF_INFLOW_LOG && s.nonuniform)
        dispatch(res_of(s), [](uint3 id) { ref_init::CSSetLogVelBndCondNonUniform(id); });
    else if (s.cfg.inflow_type == WF_INFLOW_LOG)
        dispatch(res_of(s), [](uint3 id) { ref_init::CSSetLogVelBndCond(id); });
    else
        dispatch(res_of(s), [](uint3 id) { ref_init::CSSetFixedValueVelBndCond(id); });
}

// The constructor's set-up, FvmSolverGpu.cs:207-221 (SolidType.Box aside).
void construct(wfr_solver& s) {
    set_uniforms(s);
    bind_init(s);
    dispatch(res_of(s), [](uint3 id) { ref_init::CSInitFlagField(id); });  // InitFlagField
    init_vel_pres_fields(s);
    if (s.cfg.turbulence == WF_TURB_SMAGORINSKY) {
        // InitFaceEddyVisField (:941-945) dispatches kernel index
        // initFaceEddyVisFieldKernel, which is never looked up and so is 0:
        // the first kernel of the shader, CSInitFlagField, over
        // (gridRes + 8) / 8 groups.  The face texture keeps its zeros.
        bind_init(s);
        dispatch(int3(s.nx + 1, s.ny + 1, s.nz + 1), [](uint3 id) { ref_init::CSInitFlagField(id); });
    }
    bind_init(s);
    dispatch(res_of(s), [](uint3 id) { ref_init::CSSetZeroVelBndCond(id); });
    set_fixed_value_vel_bnd_cond(s);
}

// Field id -> texture; vectors as float4 (xyz used), scalars as float.
float4* vec_field(wfr_solver& s, int f) {
    switch (f) {
        case WF_FIELD_VEL: return s.vel;
        case WF_FIELD_VEL_LAST_TIME: return s.velLastTime;
        case WF_FIELD_VEL_LAST_ITER: return s.velLastIter;
        case WF_FIELD_VEL_CORRECT: return s.velCorrect;
        case WF_FIELD_D: return s.D;
        case WF_FIELD_B: return s.b;
        case WF_FIELD_AODU: return s.aodu;
        case WF_FIELD_FACE_EDDY_VIS: return s.face;
        default: return nullptr;
    }
}
float* scalar_field(wfr_solver& s, int f) {
    switch (f) {
        case WF_FIELD_PRES: return s.pres;
        case WF_FIELD_PRES_CORRECT: return s.pc;
        case WF_FIELD_PRES_CORRECT_LAST_ITER: return s.pcLastIter;
        case WF_FIELD_DP: return s.Dp;
        case WF_FIELD_BP: return s.bp;
        case WF_FIELD_EDDY_VIS: return s.eddy;
        default: return nullptr;
    }
}

}  // namespace

extern "C" {

static int create(const wf_config* cfg, bool construct_fields, wfr_solver** out) {
    if (!cfg || !out || cfg->nx < 1 || cfg->ny < 1 || cfg->nz < 1) return WF_ERR_INVALID_ARG;
    if (cfg->calc_residual) return WF_ERR_UNSUPPORTED;
    if (construct_fields && cfg->inflow_ustar > 0.f) return WF_ERR_UNSUPPORTED;
    wfr_solver* s = new (std::nothrow) wfr_solver();
    if (!s) return WF_ERR_OOM;
    s->cfg = *cfg;
    s->nx = cfg->nx;
    s->ny = cfg->ny;
    s->nz = cfg->nz;
    s->n = (size_t)s->nx * s->ny * s->nz;
    // FluidSimConfig.cs:326-339: ds, dv and nu are computed in float.
    s->dx = cfg->dx;
    s->ds = cfg->dx * cfg->dx;
    s->dv = cfg->dx * cfg->dx * cfg->dx;
    s->nu = cfg->mu / cfg->den;
    for (auto& v : s->store4) v.assign(s->n, float4());
    for (auto& v : s->store1) v.assign(s->n, 0.f);
    s->bnd[WF_FACE_X0].assign((size_t)s->ny * s->nz, float4());
    s->bnd[WF_FACE_XN].assign((size_t)s->ny * s->nz, float4());
    s->bnd[WF_FACE_Y0].assign((size_t)s->nx * s->nz, float4());
    s->bnd[WF_FACE_YN].assign((size_t)s->nx * s->nz, float4());
    s->bnd[WF_FACE_Z0].assign((size_t)s->nx * s->ny, float4());
    s->bnd[WF_FACE_ZN].assign((size_t)s->nx * s->ny, float4());
    s->flag.assign(s->n, WF_CELL_FLUID);
    s->vel = s->store4[0].data();
    s->velLastTime = s->store4[1].data();
    s->velLastIter = s->store4[2].data();
    s->velCorrect = s->store4[3].data();
    s->aodu = s->store4[4].data();
    s->D = s->store4[5].data();
    s->b = s->store4[6].data();
    s->face = s->store4[7].data();
    s->pres = s->store1[0].data();
    s->pc = s->store1[1].data();
    s->pcLastIter = s->store1[2].data();
    s->Dp = s->store1[3].data();
    s->bp = s->store1[4].data();
    s->eddy = s->store1[5].data();
    s->wind = cfg->wind_speed;
    if (construct_fields) construct(*s);
    *out = s;
    return WF_OK;
}

/* Allocates the textures and runs the constructor's set-up (FvmSolverGpu.cs:
 * 173-222) with RuntimeConfig.windSpeed = cfg->wind_speed.  The inflow's
 * friction-velocity override (inflow_ustar) and residual early exit have no
 * counterpart in the reference's kernels and are rejected. */
int wfr_create(const wf_config* cfg, wfr_solver** out) { return create(cfg, true, out); }

/* Allocates the textures only (all cells fluid, every field zero), for a
 * state that the caller sets field by field. */
int wfr_create_empty(const wf_config* cfg, wfr_solver** out) { return create(cfg, false, out); }

/* InitFlags (FvmSolverGpu.cs:964-980): CSInitModelFlag over int32 flags. */
int wfr_init_flags(wfr_solver* s, const int32_t* flags, size_t n) {
    if (!s || !flags || n != s->n) return WF_ERR_INVALID_ARG;
    std::vector<int> buf(flags, flags + n);
    set_uniforms(*s);
    bind_init(*s);
    ref_init::flagFieldBuffer.p = buf.data();
    ref_init::flagFieldBuffer.n = buf.size();
    dispatch(res_of(*s), [](uint3 id) { ref_init::CSInitModelFlag(id); });
    ref_init::flagFieldBuffer.p = nullptr;
    return WF_OK;
}

/* InitVelPresFields (:786-860) with RuntimeConfig.windSpeed = wind_speed. */
int wfr_init_vel_pres_fields(wfr_solver* s, float wind_speed) {
    if (!s) return WF_ERR_INVALID_ARG;
    s->wind = wind_speed;
    init_vel_pres_fields(*s);
    return WF_OK;
}

/* SetFixedValueVelBndCond (:998-1022) with RuntimeConfig.windSpeed = wind_speed. */
int wfr_set_fixed_value_vel_bnd_cond(wfr_solver* s, float wind_speed) {
    if (!s) return WF_ERR_INVALID_ARG;
    s->wind = wind_speed;
    set_fixed_value_vel_bnd_cond(*s);
    return WF_OK;
}

/* InitVelPresFieldsFromBackGroundFlow (:898-929): samples bg's velField and
 * presFieldLastTime textures (the ones GetVelField / GetPresField return,
 * :1568-1577) with CSInitVelPresFieldsFromBGFlowRotate. */
int wfr_init_from_background(wfr_solver* s, const wfr_solver* bg, const float pos[3], const float pos_bg[3],
                             float rot_deg) {
    if (!s || !bg || !pos || !pos_bg) return WF_ERR_INVALID_ARG;
    set_uniforms(*s);
    bind_init(*s);
    {
        using namespace ref_init;
        dxFG = s->dx;
        dxBG = bg->dx;
        physFieldPosFG = hlsl::float3(pos[0], pos[1], pos[2]);
        physFieldPosBG = hlsl::float3(pos_bg[0], pos_bg[1], pos_bg[2]);
        fieldRotAng = rot_deg * (float)(3.1415926 / 180);
        gridResBG = int3(bg->nx, bg->ny, bg->nz);
        velFieldBG.bind(bg->vel, bg->nx, bg->ny, bg->nz);
        presFieldBG.bind(bg->pres, bg->nx, bg->ny, bg->nz);
    }
    dispatch(res_of(*s), [](uint3 id) { ref_init::CSInitVelPresFieldsFromBGFlowRotate(id); });
    return WF_OK;
}

int wfr_destroy(wfr_solver* s) {
    delete s;
    return WF_OK;
}

/* Raw flag values (WF_CELL_FLUID / WF_CELL_SOLID), n = nx*ny*nz. */
int wfr_set_flags(wfr_solver* s, const int32_t* flags, size_t n) {
    if (!s || !flags || n != s->n) return WF_ERR_INVALID_ARG;
    for (size_t i = 0; i < n; ++i) s->flag[i] = flags[i];
    return WF_OK;
}

int wfr_get_flags(wfr_solver* s, int32_t* out) {
    if (!s || !out) return WF_ERR_INVALID_ARG;
    for (size_t i = 0; i < s->n; ++i) out[i] = s->flag[i];
    return WF_OK;
}

/* Number of points of a field (cells, or boundary-plane points). */
static size_t points_of(const wfr_solver* s, int f) {
    switch (f) {
        case WF_FIELD_BND_X0:
        case WF_FIELD_BND_XN: return (size_t)s->ny * s->nz;
        case WF_FIELD_BND_Y0:
        case WF_FIELD_BND_YN: return (size_t)s->nx * s->nz;
        case WF_FIELD_BND_Z0:
        case WF_FIELD_BND_ZN: return (size_t)s->nx * s->ny;
        default: return s->n;
    }
}

/* Field transfer in the library's layout: scalars one plane, vectors three
 * SoA planes (x, y, z), boundary planes as in windfvm.h. */
int wfr_set_field(wfr_solver* s, int field, const float* in) {
    if (!s || !in) return WF_ERR_INVALID_ARG;
    if (field >= WF_FIELD_BND_X0 && field <= WF_FIELD_BND_ZN) {
        std::vector<float4>& p = s->bnd[field - WF_FIELD_BND_X0];
        const size_t m = p.size();
        for (size_t i = 0; i < m; ++i) p[i] = float4(in[i], in[m + i], in[2 * m + i], 0.f);
        return WF_OK;
    }
    if (float4* v = vec_field(*s, field)) {
        for (size_t i = 0; i < s->n; ++i) v[i] = float4(in[i], in[s->n + i], in[2 * s->n + i], 0.f);
        return WF_OK;
    }
    if (float* v = scalar_field(*s, field)) {
        std::memcpy(v, in, s->n * sizeof(float));
        return WF_OK;
    }
    return WF_ERR_INVALID_ARG;
}

int wfr_get_field(wfr_solver* s, int field, float* out) {
    if (!s || !out) return WF_ERR_INVALID_ARG;
    const float4* v = nullptr;
    size_t m = points_of(s, field);
    if (field >= WF_FIELD_BND_X0 && field <= WF_FIELD_BND_ZN)
        v = s->bnd[field - WF_FIELD_BND_X0].data();
    else
        v = vec_field(*s, field);
    if (v) {
        for (size_t i = 0; i < m; ++i) {
            out[i] = v[i].x;
            out[m + i] = v[i].y;
            out[2 * m + i] = v[i].z;
        }
        return WF_OK;
    }
    if (const float* p = scalar_field(*s, field)) {
        std::memcpy(out, p, s->n * sizeof(float));
        return WF_OK;
    }
    return WF_ERR_INVALID_ARG;
}

int wfr_step(wfr_solver* s, int n_steps) {
    if (!s || n_steps < 0) return WF_ERR_INVALID_ARG;
    for (int i = 0; i < n_steps; ++i) {
        if (s->nonuniform)
            step_once_nu(*s);
        else
            step_once(*s);
    }
    return WF_OK;
}

/* Switches the solver to the non-uniform collocated grid (gridType
 * CollNonUniform): face positions fx[nx+1], fy[ny+1], fz[nz+1], strictly
 * increasing (InitMeshBuffers, FvmSolverGpu.cs:682-788, fills the same
 * buffers from a hard-coded stretching pattern).  All three NULL returns to
 * the uniform grid.  The face-flux texture starts at zero.
 *
 * Binding.  The reference binds velFaceFluxField only for the pressure
 * pre-compute, which writes it (:1295); the two momentum kernels that read
 * it (FvmCollNonUniform.compute:204-335, 799-841) have their SetTexture calls
 * commented out (:1160, :1196).  Here the texture is bound for them too, so
 * that the momentum equation sees the face fluxes of the last pressure
 * pre-compute, the intended data flow.  SIMPLE is replayed with or without
 * the Smagorinsky model (its Les and WallFunc shaders take the constant dx on
 * every grid); PISO is refused, as InitPisoShader throws for this grid type
 * (:493-496). */
int wfr_set_face_positions(wfr_solver* s, const float* fx, const float* fy, const float* fz) {
    if (!s) return WF_ERR_INVALID_ARG;
    if (!fx && !fy && !fz) {
        s->nonuniform = false;
        return WF_OK;
    }
    if (!fx || !fy || !fz) return WF_ERR_INVALID_ARG;
    if (s->cfg.solver_type != WF_SOLVER_SIMPLE) return WF_ERR_UNSUPPORTED;
    auto ok = [](const float* f, int n) {
        for (int i = 0; i < n; ++i)
            if (!(f[i + 1] > f[i])) return false;
        return true;
    };
    if (!ok(fx, s->nx) || !ok(fy, s->ny) || !ok(fz, s->nz)) return WF_ERR_INVALID_ARG;
    s->fpx.assign(fx, fx + s->nx + 1);
    s->fpy.assign(fy, fy + s->ny + 1);
    s->fpz.assign(fz, fz + s->nz + 1);
    s->flux.assign((size_t)(s->nx + 1) * (s->ny + 1) * (s->nz + 1), hlsl::float3());
    s->nonuniform = true;
    return WF_OK;
}

/* The face-flux texture, three planes (x, y, z components) of
 * (nx+1)*(ny+1)*(nz+1) points, x fastest. */
int wfr_get_face_flux(wfr_solver* s, float* out) {
    if (!s || !out || !s->nonuniform) return WF_ERR_INVALID_ARG;
    const size_t m = s->flux.size();
    for (size_t i = 0; i < m; ++i) {
        out[i] = s->flux[i].x;
        out[m + i] = s->flux[i].y;
        out[2 * m + i] = s->flux[i].z;
    }
    return WF_OK;
}

}  // extern "C"
