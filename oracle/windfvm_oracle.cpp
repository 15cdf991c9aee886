// windfvm_oracle.cpp - CPU oracle for the collocated SIMPLE/PISO LES step.
//
// TEST INFRASTRUCTURE ONLY.  This is a plain C++17 restatement of the
// reference's HLSL kernels (puppy2333/UnityWindSimulation, paths below are
// relative to that project) and of the step sequencing of FvmSolverGpu.cs.
// It exists to check the CUDA library; nothing in the library calls it.
//
// Arithmetic follows the HLSL expression trees term by term (same operand
// order and parenthesisation), templated on R = float or double.  Build with
// -ffp-contract=off so the FP32 instance rounds like an IEEE FP32 machine
// without contraction.
//
// Field roles mirror the reference textures (FvmSolverGpu.cs:263-305): the
// three velocity buffers and the two pressure-correction buffers are swapped
// by reference exactly where the C# driver swaps them.
#include "windfvm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

template <class R> struct V3 { R c[3]; };

struct Face {
    int ox, oy, oz;  // neighbour offset
    int axis;        // 0 x, 1 y, 2 z
    int sign;        // +1 for E/N/U faces, -1 for W/S/D faces
    int bc;          // WF_FACE_* of the domain face crossed
};
// Face order E, W, N, S, U, D: the order in which every reference kernel
// accumulates its face terms.
constexpr Face kFaces[6] = {
    {+1, 0, 0, 0, +1, WF_FACE_XN}, {-1, 0, 0, 0, -1, WF_FACE_X0},
    {0, +1, 0, 1, +1, WF_FACE_YN}, {0, -1, 0, 1, -1, WF_FACE_Y0},
    {0, 0, +1, 2, +1, WF_FACE_ZN}, {0, 0, -1, 2, -1, WF_FACE_Z0}};

template <class R> struct Oracle {
    wf_config cf{};
    int nx = 0, ny = 0, nz = 0;
    size_t N = 0;
    R dx{}, ds{}, dv{}, dt{}, nu{}, den{}, cs{};
    R force[3]{};
    float wind = 0.f;
    bool les = false;

    std::vector<int32_t> flag;
    std::vector<V3<R>> vel, velT, velI, velC, Dv, bv, aodu, face;
    std::vector<R> p, pc, pcL, Dp, bp, eddy;
    std::vector<R> drag;  // Brinkman drag per cell (library extension; zero = reference equations)
    std::vector<V3<R>> bnd[6];
    int64_t step = 0;
    double res_vel = -1.0, res_pres = -1.0;

    // ---------------------------------------------------------------- helpers
    size_t idx(int x, int y, int z) const { return (size_t(z) * ny + y) * nx + x; }
    bool in_region(int x, int y, int z) const {
        return x >= 0 && x < nx && y >= 0 && y < ny && z >= 0 && z < nz;
    }
    bool fluid(int x, int y, int z) const { return flag[idx(x, y, z)] == WF_CELL_FLUID; }
    bool in_fluid(int x, int y, int z) const { return in_region(x, y, z) && fluid(x, y, z); }
    bool in_solid(int x, int y, int z) const {
        return in_region(x, y, z) && flag[idx(x, y, z)] == WF_CELL_SOLID;
    }
    size_t plane_idx(int bc, int x, int y, int z) const {
        if (bc <= WF_FACE_XN) return size_t(z) * ny + y;  // bndFieldX*[int2(y, z)]
        if (bc <= WF_FACE_YN) return size_t(z) * nx + x;  // bndFieldY*[int2(x, z)]
        return size_t(y) * nx + x;                        // bndFieldZ*[int2(x, y)]
    }
    const V3<R>& bndv(int bc, int x, int y, int z) const { return bnd[bc][plane_idx(bc, x, y, z)]; }
    // faceEddyVisField read.  With WF_COMPAT_RFLOAT_FACE_EDDY_VIS the texture
    // is single-channel, so .y/.z read back as 0 (FvmSolverGpu.cs:304).
    R face_read(size_t i, int axis) const {
        if ((cf.compat_flags & WF_COMPAT_RFLOAT_FACE_EDDY_VIS) && axis != 0) return R(0);
        return face[i].c[axis];
    }
    template <class F> void for_cells(F&& fn) {
#pragma omp parallel for schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) fn(x, y, z);
    }

    // Face viscosity nu + nu_t on face f of fluid cell P, FvmColl.compute:1596-1635
    // (same block in CSVelPredict :1962-2001 and LES.compute:643-679).
    R vis_face(int x, int y, int z, int f) const {
        if (!les) return nu;
        const Face& F = kFaces[f];
        const size_t P = idx(x, y, z);
        int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
        R v = nu + eddy[P];
        if (in_fluid(X, Y, Z)) {
            v = nu + R(0.5) * (eddy[P] + eddy[idx(X, Y, Z)]);
        } else if (in_solid(X, Y, Z)) {
            // E/N/U faces are stored at the neighbour's W/S/D slot.
            size_t i = F.sign > 0 ? idx(X, Y, Z) : P;
            v = nu + face_read(i, F.axis);
        } else if (f == 3 && !in_region(X, Y, Z) && cf.vel_bc[WF_FACE_Y0] == WF_BND_FIXED_VALUE) {
            v = nu + face_read(P, 1);  // ground wall, FvmColl.compute:1623-1624
        }
        return v;
    }

    // ----------------------------------------------------------- init / BCs
    void setup(const wf_config& c) {
        cf = c;
        nx = c.nx; ny = c.ny; nz = c.nz;
        N = size_t(nx) * ny * nz;
        dx = R(c.dx);
        ds = dx * dx;                       // FluidSimConfig.cs:326
        dv = dx * dx * dx;                  // :327
        dt = R(c.dt);
        den = R(c.den);
        nu = R(float(c.mu / c.den));        // :339 (computed in float by the C# side)
        cs = R(c.cs);
        for (int i = 0; i < 3; ++i) force[i] = R(c.ext_force[i]);
        wind = c.wind_speed;
        les = c.turbulence == WF_TURB_SMAGORINSKY;
        V3<R> z3{{R(0), R(0), R(0)}};
        flag.assign(N, WF_CELL_FLUID);  // CSInitFlagField, InitShaderColl.compute:84-92
        vel.assign(N, z3); velT.assign(N, z3); velI.assign(N, z3); velC.assign(N, z3);
        Dv.assign(N, z3); bv.assign(N, z3); aodu.assign(N, z3); face.assign(N, z3);
        p.assign(N, R(0)); pc.assign(N, R(0)); pcL.assign(N, R(0));
        Dp.assign(N, R(0)); bp.assign(N, R(0)); eddy.assign(N, R(0)); drag.assign(N, R(0));
        bnd[0].assign(size_t(ny) * nz, z3); bnd[1].assign(size_t(ny) * nz, z3);
        bnd[2].assign(size_t(nx) * nz, z3); bnd[3].assign(size_t(nx) * nz, z3);
        bnd[4].assign(size_t(nx) * ny, z3); bnd[5].assign(size_t(nx) * ny, z3);
        // Constructor order, FvmSolverGpu.cs:207-221.  faceEddyVis stays 0:
        // InitFaceEddyVisField dispatches kernel 0 (:941-945).
        init_vel_pres_fields();
        set_zero_vel_bnd_cond();
        set_fixed_value_vel_bnd_cond(wind);
    }

    // u* for the log profile: CSInitLogVelPresFields :121 / CSSetLogVelBndCond :280
    R fric_vel() const {
        if (cf.inflow_ustar > 0.f) return R(cf.inflow_ustar);
        R k = R(cf.inflow_kappa), z0 = R(cf.inflow_z0), href = R(cf.inflow_href);
        return k * R(wind) / std::log((href + z0) / z0);
    }
    R log_profile(R yPhys) const {
        R k = R(cf.inflow_kappa), z0 = R(cf.inflow_z0);
        return fric_vel() / k * std::log((yPhys + z0) / z0);
    }

    // CSInitVelPresFields / CSInitLogVelPresFields, InitShaderColl.compute:95-132.
    // Every cell (solid included) is written, as in the reference.
    void init_vel_pres_fields() {
        const bool logp = cf.inflow_type == WF_INFLOW_LOG;
        const bool centre = (cf.compat_flags & WF_COMPAT_INIT_PROFILE_CELL_CENTRE) != 0;
        for_cells([&](int x, int y, int z) {
            size_t P = idx(x, y, z);
            V3<R> u{{R(wind), R(0), R(0)}};
            if (logp) {
                R yPhys = nonuniform ? nu_centre_height(y) : centre ? (R(y) + R(0.5)) * dx : R(y) * dx;
                u = V3<R>{{log_profile(yPhys), R(0), R(0)}};
            }
            vel[P] = u; velT[P] = u; velI[P] = u;
            velC[P] = V3<R>{{R(0), R(0), R(0)}};
            p[P] = R(0); pc[P] = R(0); pcL[P] = R(0);
        });
    }
    // CSInitVelPresFieldsFromBGFlowRotate, InitShaderColl.compute:185-226
    // (host side FvmSolverGpu.cs:898-929): cell (index - res/2) * dx rotated
    // by theta about the vertical axis, placed at pos, mapped into the
    // background's frame and sampled trilinearly with clamped addressing;
    // the vector is copied unrotated.  Every cell is written.
    void init_from_background(const Oracle<R>& bg, const float pos[3], const float posb[3], float rot_deg) {
        const R th = R(rot_deg) * R(3.1415926 / 180);
        const R s1 = std::sin(th), c1 = std::cos(th), s2 = std::sin(-th), c2 = std::cos(-th);
        const int bnx = bg.nx, bny = bg.ny, bnz = bg.nz;
        auto sample = [&](auto get, R u, R v, R w) {
            const R tx = u * R(bnx) - R(0.5), ty = v * R(bny) - R(0.5), tz = w * R(bnz) - R(0.5);
            const R fx = std::floor(tx), fy = std::floor(ty), fz = std::floor(tz);
            const R ax = tx - fx, ay = ty - fy, az = tz - fz;
            auto cl = [](int i, int n) { return i < 0 ? 0 : (i > n - 1 ? n - 1 : i); };
            const int x0 = cl(int(fx), bnx), x1 = cl(int(fx) + 1, bnx);
            const int y0 = cl(int(fy), bny), y1 = cl(int(fy) + 1, bny);
            const int z0 = cl(int(fz), bnz), z1 = cl(int(fz) + 1, bnz);
            const R c00 = get(x0, y0, z0) * (R(1) - ax) + get(x1, y0, z0) * ax;
            const R c10 = get(x0, y1, z0) * (R(1) - ax) + get(x1, y1, z0) * ax;
            const R c01 = get(x0, y0, z1) * (R(1) - ax) + get(x1, y0, z1) * ax;
            const R c11 = get(x0, y1, z1) * (R(1) - ax) + get(x1, y1, z1) * ax;
            const R c0 = c00 * (R(1) - ay) + c10 * ay;
            const R c1 = c01 * (R(1) - ay) + c11 * ay;
            return c0 * (R(1) - az) + c1 * az;
        };
        for_cells([&](int x, int y, int z) {
            const R lx = R(x - nx / 2) * dx, ly = R(y - ny / 2) * dx, lz = R(z - nz / 2) * dx;
            const R gx = R(pos[0]) + (lx * c1 + lz * s1), gy = R(pos[1]) + ly, gz = R(pos[2]) + (lz * c1 - lx * s1);
            const R rx = gx - R(posb[0]), ry = gy - R(posb[1]), rz = gz - R(posb[2]);
            const R bx = rx * c2 + rz * s2, by = ry, bz = rz * c2 - rx * s2;
            const R u = bx / (R(bnx) * bg.dx) + R(0.5);
            const R v = by / (R(bny) * bg.dx) + R(0.5);
            const R w = bz / (R(bnz) * bg.dx) + R(0.5);
            V3<R> uu;
            for (int k = 0; k < 3; ++k)
                uu.c[k] = sample([&](int X, int Y, int Z) { return bg.velT[bg.idx(X, Y, Z)].c[k]; }, u, v, w);
            const size_t P = idx(x, y, z);
            vel[P] = uu; velT[P] = uu; velI[P] = uu;
            velC[P] = V3<R>{{R(0), R(0), R(0)}};
            p[P] = sample([&](int X, int Y, int Z) { return bg.p[bg.idx(X, Y, Z)]; }, u, v, w);
            pc[P] = R(0); pcL[P] = R(0);
        });
    }
    // CSSetZeroVelBndCond, InitShaderColl.compute:229-248
    void set_zero_vel_bnd_cond() {
        for (auto& b : bnd) std::fill(b.begin(), b.end(), V3<R>{{R(0), R(0), R(0)}});
    }
    // CSSetFixedValueVelBndCond / CSSetLogVelBndCond, InitShaderColl.compute:253-285
    void set_fixed_value_vel_bnd_cond(float w) {
        wind = w;
        if (cf.inflow_type == WF_INFLOW_LOG) {
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y) {
                    R yPhys = nonuniform ? nu_centre_height(y) : (R(y) + R(0.5)) * dx;
                    bnd[WF_FACE_X0][size_t(z) * ny + y] = V3<R>{{log_profile(yPhys), R(0), R(0)}};
                }
        } else {
            for (int z = 0; z < nz; ++z)
                for (int y = 0; y < ny; ++y)
                    bnd[WF_FACE_X0][size_t(z) * ny + y] = V3<R>{{R(w), R(0), R(0)}};
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x)
                    bnd[WF_FACE_ZN][size_t(y) * nx + x] =
                        V3<R>{{R(cf.vel_zn[0]), R(cf.vel_zn[1]), R(cf.vel_zn[2])}};
        }
    }
    // CSInitModelFlag, InitShaderColl.compute:346-364
    void init_flags(const int32_t* f) {
        for_cells([&](int x, int y, int z) {
            size_t P = idx(x, y, z);
            if (double(f[P]) > 0.5) {
                flag[P] = WF_CELL_SOLID;
                V3<R> z3{{R(0), R(0), R(0)}};
                vel[P] = z3; velI[P] = z3; velT[P] = z3;
            } else {
                flag[P] = WF_CELL_FLUID;
            }
        });
    }

    // ------------------------------------------------------- wall function
    // LogLawWallFunc, WallFunc.compute:77-123
    static R log_law(R uP, R dx_, R nu_, R den_) {
        const R E = R(9.8f), k = R(0.41f);
        R C = E * (dx_ / R(2.0)) / nu_;
        R eddyVis = R(0);
        R uTau = R(1.0f);
        uP = std::fabs(uP);
        if (uP < R(1e-5f)) {
            uTau = R(0);
        } else {
            for (int i = 0; i < 10; ++i) {
                R f = uTau * std::log(C * uTau) - k * uP;
                R df = std::log(C * uTau) + R(1.0f);
                if (std::fabs(df) < R(1e-6f)) break;
                uTau = uTau - f / df;
                if (uTau < R(1e-5f)) uTau = R(1e-5f);
            }
            R tauWall = uTau * uTau * den_;
            R strainRate = uP / (dx_ / R(2.0));
            eddyVis = tauWall / (strainRate * den_) - nu_;
            if (eddyVis < R(0)) eddyVis = R(0);
        }
        return eddyVis;
    }
    // CSCalLogLawWallFunc, WallFunc.compute:128-190
    void op_wallfunc() {
        for_cells([&](int x, int y, int z) {
            size_t P = idx(x, y, z);
            R fe[3] = {R(0), R(0), R(0)};
            auto mag2 = [](R a, R b) { return std::sqrt(a * a + b * b); };
            if (fluid(x, y, z)) {
                if (in_solid(x - 1, y, z)) {
                    const V3<R>& u = velT[P];
                    fe[0] += log_law(mag2(u.c[1], u.c[2]), dx, nu, den);
                }
                if (in_solid(x, y - 1, z) ||
                    (!in_region(x, y - 1, z) && cf.vel_bc[WF_FACE_Y0] == WF_BND_FIXED_VALUE)) {
                    const V3<R>& u = velT[P];
                    fe[1] += log_law(mag2(u.c[0], u.c[2]), dx, nu, den);
                }
                if (in_solid(x, y, z - 1)) {
                    const V3<R>& u = velT[P];
                    fe[2] += log_law(mag2(u.c[0], u.c[1]), dx, nu, den);
                }
            } else if (flag[P] == WF_CELL_SOLID) {
                if (in_fluid(x - 1, y, z)) {
                    const V3<R>& u = velT[idx(x - 1, y, z)];
                    fe[0] += log_law(mag2(u.c[1], u.c[2]), dx, nu, den);
                }
                if (in_fluid(x, y - 1, z)) {
                    const V3<R>& u = velT[idx(x, y - 1, z)];
                    fe[1] += log_law(mag2(u.c[0], u.c[2]), dx, nu, den);
                }
                if (in_fluid(x, y, z - 1)) {
                    const V3<R>& u = velT[idx(x, y, z - 1)];
                    fe[2] += log_law(mag2(u.c[0], u.c[1]), dx, nu, den);
                }
            }
            face[P] = V3<R>{{fe[0], fe[1], fe[2]}};
        });
    }

    // ---------------------------------------------------------------- LES
    // Get{E,W,N,S,U,D}FaceVelLastTime, LES.compute:104-258
    V3<R> face_vel(int x, int y, int z, int f) const {
        const Face& F = kFaces[f];
        int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
        const V3<R>& u = velT[idx(x, y, z)];
        V3<R> r{{R(0), R(0), R(0)}};
        if (in_region(X, Y, Z)) {
            if (fluid(X, Y, Z)) {
                const V3<R>& v = velT[idx(X, Y, Z)];
                for (int c = 0; c < 3; ++c) r.c[c] = R(0.5) * (u.c[c] + v.c[c]);
            }
        } else {
            int bt = cf.vel_bc[F.bc];
            if (bt == WF_BND_FIXED_VALUE) {
                r = bndv(F.bc, x, y, z);
            } else if (bt == WF_BND_ZERO_GRAD) {
                r = u;
            } else if (bt == WF_BND_SYMMETRY) {
                r = u;
                r.c[F.axis] = R(0);
            }
        }
        return r;
    }
    // Cell-centre velocity gradient g[i][j] = d u_i / d x_j (LES.compute:296-306)
    void cell_grad(int x, int y, int z, R g[3][3]) const {
        V3<R> fv[6];
        for (int f = 0; f < 6; ++f) fv[f] = face_vel(x, y, z, f);
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) g[i][j] = (fv[2 * j].c[i] - fv[2 * j + 1].c[i]) / dx;
    }
    // CSCalEddyVis, LES.compute:268-324
    void op_eddy_vis() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            R g[3][3];
            cell_grad(x, y, z, g);
            R Sxx = g[0][0], Syy = g[1][1], Szz = g[2][2];
            R Sxy = R(0.5f) * (g[0][1] + g[1][0]);
            R Syz = R(0.5f) * (g[1][2] + g[2][1]);
            R Szx = R(0.5f) * (g[2][0] + g[0][2]);
            R Sabs = std::sqrt(R(2.0f) * (Sxx * Sxx + Syy * Syy + Szz * Szz + R(2.0f) * Sxy * Sxy +
                                          R(2.0f) * Syz * Syz + R(2.0f) * Szx * Szx));
            eddy[idx(x, y, z)] = (cs * cs) * (dx * dx) * Sabs;
        });
    }
    // CSCalLesDeferCorrectTerm, LES.compute:327-687.  Writes bField.
    void op_les_term() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            R g[3][3];
            cell_grad(x, y, z, g);
            // fg[f][j]: on face f, d u_a / d x_j with a = the face's axis.
            R fg[6][3] = {};
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int a = F.axis;
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    if (fluid(X, Y, Z)) {
                        R gn[3][3];
                        cell_grad(X, Y, Z, gn);
                        for (int j = 0; j < 3; ++j) fg[f][j] = R(0.5) * (g[a][j] + gn[a][j]);
                    } else {
                        // e.g. eFacePuxpx = -u_P.x / (0.5 dx); wFacePuxpx = u_P.x / (0.5 dx)
                        R v = velT[P].c[a] / (R(0.5) * dx);
                        fg[f][a] = F.sign > 0 ? -v : v;
                    }
                } else {
                    int bt = cf.vel_bc[F.bc];
                    if (bt == WF_BND_FIXED_VALUE) {
                        R b = bndv(F.bc, x, y, z).c[a];
                        R u = velT[P].c[a];
                        fg[f][a] = F.sign > 0 ? (b - u) / (R(0.5) * dx) : (u - b) / (R(0.5) * dx);
                    } else if (bt == WF_BND_ZERO_GRAD || bt == WF_BND_SYMMETRY) {
                        for (int j = 0; j < 3; ++j)
                            if (j != a) fg[f][j] = g[a][j];
                    }
                }
            }
            R vis[6];
            for (int f = 0; f < 6; ++f) vis[f] = vis_face(x, y, z, f);
            V3<R> out;
            for (int j = 0; j < 3; ++j) {
                // ds * (visE*e - visW*w + visN*n - visS*s + visU*u - visD*d)
                R t = vis[0] * fg[0][j] - vis[1] * fg[1][j] + vis[2] * fg[2][j] - vis[3] * fg[3][j] +
                      vis[4] * fg[4][j] - vis[5] * fg[5][j];
                out.c[j] = ds * t;
            }
            bv[P] = out;
        });
    }

    // ------------------------------------------- non-uniform collocated grid
    // gridType CollNonUniform (FvmSolverGpu.cs:185-205): face positions
    // facePosX/Y/Z (InitMeshBuffers, :682-788) and the face-flux texture
    // velFaceFluxField ((nx+1)(ny+1)(nz+1) texels, :275) that the pressure
    // pre-compute writes and the momentum kernels read (bound for them here;
    // the reference's SetTexture calls for them are commented out,
    // :1160,1196).  Restates FvmCollNonUniform.compute term by term; SIMPLE
    // without turbulence only.
    bool nonuniform = false;
    std::vector<R> fpx, fpy, fpz;
    std::vector<V3<R>> flux;
    size_t fidx(int x, int y, int z) const { return (size_t(z) * (ny + 1) + y) * (nx + 1) + x; }
    // Spacing of cell i and its neighbours along one axis; a neighbour outside
    // the domain takes the cell's own spacing (:130-142, :954-977).
    struct Sp {
        R d, dp, dm, dpp, dmm;
    };
    static Sp spacing(const std::vector<R>& f, int i, int n) {
        Sp s;
        s.d = f[i + 1] - f[i];
        s.dp = i + 1 < n ? f[i + 2] - f[i + 1] : s.d;
        s.dm = i > 0 ? f[i] - f[i - 1] : s.d;
        s.dpp = i + 2 < n ? f[i + 3] - f[i + 2] : s.d;
        s.dmm = i > 1 ? f[i - 1] - f[i - 2] : s.d;
        return s;
    }
    struct Geo {
        Sp s[3];
        R ds[3], dv;
    };
    Geo geo(int x, int y, int z) const {
        Geo g;
        g.s[0] = spacing(fpx, x, nx);
        g.s[1] = spacing(fpy, y, ny);
        g.s[2] = spacing(fpz, z, nz);
        const R dX = g.s[0].d, dY = g.s[1].d, dZ = g.s[2].d;
        g.ds[0] = dY * dZ;  // dsx
        g.ds[1] = dX * dZ;  // dsy
        g.ds[2] = dX * dY;  // dsz
        g.dv = dX * dY * dZ;
        return g;
    }
    // Own-cell interpolation weight at face f: wPe = dxE / (dx + dxE) etc.
    static R w_self(const Geo& g, int f) {
        const Sp& s = g.s[kFaces[f].axis];
        const R dq = kFaces[f].sign > 0 ? s.dp : s.dm;
        return dq / (s.d + dq);
    }
    // Centre distance across face f: 0.5 * dx + 0.5 * dxE etc.
    static R h_face(const Geo& g, int f) {
        const Sp& s = g.s[kFaces[f].axis];
        return R(0.5) * s.d + R(0.5) * (kFaces[f].sign > 0 ? s.dp : s.dm);
    }
    // velFaceFluxField read of face f: the neighbour's texel for E/N/U, the
    // cell's own for W/S/D.
    R face_flux(int x, int y, int z, int f) const {
        const Face& F = kFaces[f];
        const size_t t = F.sign > 0 ? fidx(x + F.ox, y + F.oy, z + F.oz) : fidx(x, y, z);
        return flux[t].c[F.axis];
    }

    // Face viscosities of the non-uniform momentum kernels (FvmCollNonUniform.
    // compute:483-505, same block in CSVelPredict :846-868): nu without LES;
    // with useLES nu + nu_t,P, and nu + wP nu_t,P + wQ nu_t,Q across a face to
    // a fluid neighbour, with the linear interpolation weights of the mesh.
    void nu_face_vis(int x, int y, int z, const Geo& g, R vis[6]) const {
        for (int f = 0; f < 6; ++f) vis[f] = nu;
        if (!les) return;
        const size_t P = idx(x, y, z);
        for (int f = 0; f < 6; ++f) vis[f] = nu + eddy[P];
        for (int f = 0; f < 6; ++f) {
            const Face& F = kFaces[f];
            const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
            if (!in_fluid(X, Y, Z)) continue;
            const R wP = w_self(g, f), wQ = R(1.0f) - wP;
            vis[f] = nu + wP * eddy[P] + wQ * eddy[idx(X, Y, Z)];
        }
    }

    // CSVelPredictPreCompute, FvmCollNonUniform.compute:111-721.
    void nu_vel_precompute() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            const Geo g = geo(x, y, z);
            R D[3] = {g.dv / dt, g.dv / dt, g.dv / dt};
            R b[3] = {R(0), R(0), R(0)};
            // advection, :200-335
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int a = F.axis;
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_fluid(X, Y, Z)) {
                    const R t = g.ds[a] * w_self(g, f) * face_flux(x, y, z, f);
                    for (int k = 0; k < 3; ++k) D[k] = F.sign > 0 ? D[k] + t : D[k] - t;
                } else if (!in_region(X, Y, Z)) {
                    const int bt = cf.vel_bc[F.bc];
                    const R Fv = face_flux(x, y, z, f);
                    if (bt == WF_BND_FIXED_VALUE) {
                        const V3<R>& bb = bndv(F.bc, x, y, z);
                        for (int k = 0; k < 3; ++k) {
                            const R t = g.ds[a] * bb.c[k] * Fv;
                            b[k] = F.sign > 0 ? b[k] - t : b[k] + t;
                        }
                    } else if (bt == WF_BND_ZERO_GRAD) {
                        const R t = g.ds[a] * Fv;
                        for (int k = 0; k < 3; ++k) D[k] = F.sign > 0 ? D[k] + t : D[k] - t;
                    }
                }
            }
            // pressure, :337-466
            R pf[6];
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    if (fluid(X, Y, Z)) {
                        const R wP = w_self(g, f), wQ = R(1.0f) - wP;
                        pf[f] = wP * p[P] + wQ * p[idx(X, Y, Z)];
                    } else {
                        pf[f] = p[P];
                    }
                } else {
                    pf[f] = cf.pres_bc[F.bc] == WF_BND_FIXED_VALUE ? R(0) : p[P];
                }
            }
            for (int a = 0; a < 3; ++a) b[a] += -(R(1.0) / den) * g.ds[a] * (pf[2 * a] - pf[2 * a + 1]);
            // diffusion, :468-697
            R visf[6];
            nu_face_vis(x, y, z, g, visf);
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int a = F.axis;
                const R vis = visf[f];
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    const R t = fluid(X, Y, Z) ? vis * g.ds[a] / h_face(g, f)
                                               : vis * g.ds[a] / (R(0.5) * g.s[a].d);
                    for (int k = 0; k < 3; ++k) D[k] += t;
                } else {
                    const int bt = cf.vel_bc[F.bc];
                    if (bt == WF_BND_FIXED_VALUE) {
                        const V3<R>& bb = bndv(F.bc, x, y, z);
                        for (int k = 0; k < 3; ++k) b[k] += vis * g.ds[a] / (R(0.5) * g.s[a].d) * bb.c[k];
                        for (int k = 0; k < 3; ++k) D[k] += vis * g.ds[a] / (R(0.5) * g.s[a].d);
                    } else if (bt == WF_BND_SYMMETRY) {
                        D[a] += vis * g.ds[a] / (R(0.5) * g.s[a].d);
                    }
                }
            }
            // time and force, :699-710
            for (int k = 0; k < 3; ++k) b[k] += g.dv / dt * velT[P].c[k];
            for (int k = 0; k < 3; ++k) b[k] += g.dv * force[k];
            // LES deferred-correction term, :712-717
            if (les)
                for (int k = 0; k < 3; ++k) b[k] += bv[P].c[k];
            Dv[P] = V3<R>{{D[0], D[1], D[2]}};
            bv[P] = V3<R>{{b[0], b[1], b[2]}};
        });
    }
    // CSVelPredict, FvmCollNonUniform.compute:725-917.
    void nu_vel_sweep() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            const Geo g = geo(x, y, z);
            R adv[3] = {R(0), R(0), R(0)}, dif[3] = {R(0), R(0), R(0)};
            for (int f = 0; f < 6; ++f) {  // :797-842
                const Face& F = kFaces[f];
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) continue;
                const R wQ = R(1.0f) - w_self(g, f);
                const R Fv = face_flux(x, y, z, f);
                const V3<R>& uQ = velI[idx(X, Y, Z)];
                for (int k = 0; k < 3; ++k) {
                    const R t = g.ds[F.axis] * wQ * uQ.c[k] * Fv;
                    adv[k] = F.sign > 0 ? adv[k] - t : adv[k] + t;
                }
            }
            R visf[6];
            nu_face_vis(x, y, z, g, visf);
            for (int f = 0; f < 6; ++f) {  // :844-907
                const Face& F = kFaces[f];
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) continue;
                const V3<R>& uQ = velI[idx(X, Y, Z)];
                for (int k = 0; k < 3; ++k) dif[k] += visf[f] * g.ds[F.axis] / h_face(g, f) * uQ.c[k];
            }
            V3<R> u;
            for (int k = 0; k < 3; ++k) u.c[k] = R(1.0) / Dv[P].c[k] * (adv[k] + dif[k] + bv[P].c[k]);
            vel[P] = u;
        });
    }
    // CSPresCorrectRhieChowPreCompute, FvmCollNonUniform.compute:920-1344.
    void nu_pres_precompute() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            const Geo g = geo(x, y, z);
            R dp = R(0), b = R(0);
            R uf[6] = {R(0), R(0), R(0), R(0), R(0), R(0)};
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int a = F.axis;
                const Sp& s = g.s[a];
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    if (!fluid(X, Y, Z)) continue;  // solid neighbour: no flux
                    const size_t Q = idx(X, Y, Z);
                    const R wP = w_self(g, f), wQ = R(1.0f) - wP;
                    const R DInv = wP * (R(1) / Dv[P].c[a]) + wQ * (R(1) / Dv[Q].c[a]);
                    const R h2 = h_face(g, f);
                    dp -= (g.dv / den) * DInv / h2;
                    R v = wP * vel[P].c[a] + wQ * vel[Q].c[a];
                    const R pP = p[P], pQ = p[Q];
                    const R grad = F.sign > 0 ? (pQ - pP) / h2 : (pP - pQ) / h2;
                    const int X2 = x + 2 * F.ox, Y2 = y + 2 * F.oy, Z2 = z + 2 * F.oz;
                    const int Xr = x - F.ox, Yr = y - F.oy, Zr = z - F.oz;
                    const bool fqq = in_fluid(X2, Y2, Z2), fr = in_fluid(Xr, Yr, Zr);
                    R ave;
                    if (F.sign > 0) {  // :1011-1020 (E), :1121-1130 (N), :1231-1240 (U)
                        const R h = s.d, hQ = s.dp, hQQ = s.dpp, hR = s.dm;
                        if (fqq && fr)
                            ave = R(0.5) * ((p[idx(X2, Y2, Z2)] - pP) / (R(0.5) * hQQ + hQ + R(0.5) * h) +
                                            (pQ - p[idx(Xr, Yr, Zr)]) / (R(0.5) * hQ + h + R(0.5) * hR));
                        else if (fqq)
                            ave = R(0.5) * ((p[idx(X2, Y2, Z2)] - pP) / (R(0.5) * hQQ + hQ + R(0.5) * h) +
                                            (pQ - pP) / (R(0.5) * hQ + R(1.5) * h));
                        else if (fr)
                            ave = R(0.5) * ((pQ - pP) / (R(1.5) * hQ + R(0.5) * h) +
                                            (pQ - p[idx(Xr, Yr, Zr)]) / (R(0.5) * hQ + h + R(0.5) * hR));
                        else
                            ave = grad;
                    } else {  // :1066-1075 (W), :1176-1185 (S), :1298-1305 (D)
                        const R h = s.d, hQ = s.dm, hQQ = s.dmm, hR = s.dp;
                        if (fqq && fr)
                            ave = R(0.5) * ((p[idx(Xr, Yr, Zr)] - pQ) / (R(0.5) * hR + h + R(0.5) * hQ) +
                                            (pP - p[idx(X2, Y2, Z2)]) / (R(0.5) * h + hQ + R(0.5) * hQQ));
                        else if (fqq)
                            ave = R(0.5) * ((pP - pQ) / (R(1.5) * h + R(0.5) * hQ) +
                                            (pP - p[idx(X2, Y2, Z2)]) / (R(0.5) * h + hQ + R(0.5) * hQQ));
                        else if (fr)
                            ave = R(0.5) * ((p[idx(Xr, Yr, Zr)] - pQ) / (R(0.5) * hR + h + R(0.5) * hQ) +
                                            (pP - pQ) / (R(0.5) * h + R(1.5) * hQ));
                        else
                            ave = grad;
                    }
                    v -= (g.dv * DInv) / den * (grad - ave);
                    uf[f] = v;
                    b = F.sign > 0 ? b + v : b - v;
                } else {
                    const int vb = cf.vel_bc[F.bc];
                    if (vb == WF_BND_FIXED_VALUE) {
                        const R v = bndv(F.bc, x, y, z).c[a];
                        uf[f] = v;
                        b = F.sign > 0 ? b + v : b - v;
                    } else if (vb == WF_BND_ZERO_GRAD) {
                        const R v = vel[P].c[a];
                        uf[f] = v;
                        b = F.sign > 0 ? b + v : b - v;
                    }
                    if (cf.pres_bc[F.bc] == WF_BND_FIXED_VALUE) {
                        const R DInv = R(1) / Dv[P].c[a];
                        dp -= (g.dv / den) * DInv / (R(0.5) * s.d);
                    }
                }
            }
            // :1335-1341
            flux[fidx(x, y, z)] = V3<R>{{uf[1], uf[3], uf[5]}};
            if (x + 1 == nx) flux[fidx(x + 1, y, z)] = V3<R>{{uf[0], R(0), R(0)}};
            if (y + 1 == ny) flux[fidx(x, y + 1, z)] = V3<R>{{R(0), uf[2], R(0)}};
            if (z + 1 == nz) flux[fidx(x, y, z + 1)] = V3<R>{{R(0), R(0), uf[4]}};
            Dp[P] = dp;
            bp[P] = b;
        });
    }
    // CSPresCorrectRhieChow, FvmCollNonUniform.compute:1346-1452.
    void nu_pres_sweep() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            const Geo g = geo(x, y, z);
            R t = R(0);
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) continue;
                const size_t Q = idx(X, Y, Z);
                const R wP = w_self(g, f), wQ = R(1.0f) - wP;
                const R DInv = wP * (R(1) / Dv[P].c[F.axis]) + wQ * (R(1) / Dv[Q].c[F.axis]);
                t -= (g.dv / den) * DInv / h_face(g, f) * pcL[Q];
            }
            pc[P] = (R(1) / Dp[P]) * (t + bp[P]);
        });
    }
    // CSApplyVelCorrectionDivergenceTheorem, FvmCollNonUniform.compute:1487-1731.
    void nu_apply_vel() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            const Geo g = geo(x, y, z);
            R pf[6];
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    if (fluid(X, Y, Z)) {
                        const R wP = w_self(g, f), wQ = R(1.0f) - wP;
                        pf[f] = wP * pc[P] + wQ * pc[idx(X, Y, Z)];
                    } else {
                        pf[f] = pc[P];
                    }
                } else {
                    pf[f] = cf.pres_bc[F.bc] == WF_BND_FIXED_VALUE ? R(0) : pc[P];
                }
            }
            V3<R> corr;
            for (int a = 0; a < 3; ++a)
                corr.c[a] = -(g.dv / den) * (R(1) / Dv[P].c[a]) * (pf[2 * a] - pf[2 * a + 1]) / g.s[a].d;
            velC[P] = corr;
            for (int a = 0; a < 3; ++a) vel[P].c[a] += corr.c[a];
        });
    }
    // CSInitLogVelPresFieldsNonUniform / CSSetLogVelBndCondNonUniform
    // (InitShaderColl.compute:134-154, 287-300): the log profile at the cell
    // centre height 0.5 (fy[y] + fy[y+1]).
    R nu_centre_height(int y) const { return R(0.5) * (fpy[y] + fpy[y + 1]); }

    // ------------------------------------------------ momentum predictor
    // CSVelPredictPreCompute, FvmColl.compute:1292-1859.  bField holds the
    // LES term on entry (when LES is on) and b on exit.
    void op_vel_precompute() {
        if (nonuniform) return nu_vel_precompute();
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            const V3<R>& uP = velT[P];
            R D[3] = {dv / dt, dv / dt, dv / dt};
            R b[3] = {R(0), R(0), R(0)};
            // Advection (CDS, Picard), :1314-1482
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int a = F.axis;
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    if (fluid(X, Y, Z)) {
                        R t = ds * R(0.25) * (uP.c[a] + velT[idx(X, Y, Z)].c[a]);
                        for (int c = 0; c < 3; ++c) D[c] = F.sign > 0 ? D[c] + t : D[c] - t;
                    }
                } else {
                    int bt = cf.vel_bc[F.bc];
                    if (bt == WF_BND_FIXED_VALUE) {
                        const V3<R>& bb = bndv(F.bc, x, y, z);
                        for (int c = 0; c < 3; ++c) {
                            R t = ds * bb.c[c] * bb.c[a];
                            b[c] = F.sign > 0 ? b[c] - t : b[c] + t;
                        }
                    } else if (bt == WF_BND_ZERO_GRAD) {
                        R t = ds * uP.c[a];
                        for (int c = 0; c < 3; ++c) D[c] = F.sign > 0 ? D[c] + t : D[c] - t;
                    }
                }
            }
            // Pressure gradient from face pressures, :1484-1591
            R pf[6];
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    pf[f] = fluid(X, Y, Z) ? R(0.5) * (p[P] + p[idx(X, Y, Z)]) : p[P];
                } else {
                    pf[f] = cf.pres_bc[F.bc] == WF_BND_FIXED_VALUE ? R(0) : p[P];
                }
            }
            for (int a = 0; a < 3; ++a) b[a] += -(R(1.0) / den) * ds * (pf[2 * a] - pf[2 * a + 1]);
            // Diffusion, :1593-1836
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                R vis = vis_face(x, y, z, f);
                if (in_region(X, Y, Z)) {
                    if (fluid(X, Y, Z)) {
                        for (int c = 0; c < 3; ++c) D[c] += vis * ds / dx;
                    } else {
                        for (int c = 0; c < 3; ++c) D[c] += R(2) * vis * ds / dx;
                    }
                } else {
                    int bt = cf.vel_bc[F.bc];
                    if (bt == WF_BND_FIXED_VALUE) {
                        const V3<R>& bb = bndv(F.bc, x, y, z);
                        for (int c = 0; c < 3; ++c) b[c] += R(2) * vis * ds / dx * bb.c[c];
                        for (int c = 0; c < 3; ++c) D[c] += R(2) * vis * ds / dx;
                    } else if (bt == WF_BND_SYMMETRY) {
                        D[F.axis] += R(2) * vis * ds / dx;
                    }
                }
            }
            // Time, force and LES terms, :1838-1854
            for (int c = 0; c < 3; ++c) b[c] += dv / dt * uP.c[c];
            for (int c = 0; c < 3; ++c) b[c] += dv * force[c];
            if (les)
                for (int c = 0; c < 3; ++c) b[c] += bv[P].c[c];
            // Brinkman drag of a soft obstacle mask (no reference counterpart)
            if (drag[P] != R(0))
                for (int c = 0; c < 3; ++c) D[c] += dv * drag[P];
            Dv[P] = V3<R>{{D[0], D[1], D[2]}};
            bv[P] = V3<R>{{b[0], b[1], b[2]}};
        });
    }
    // CSVelPredict, FvmColl.compute:1863-2069: velField <- one Jacobi sweep
    // from velFieldLastIter.
    void vel_sweep() {
        if (nonuniform) return nu_vel_sweep();
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            const V3<R>& uP = velT[P];
            R adv[3] = {R(0), R(0), R(0)}, dif[3] = {R(0), R(0), R(0)};
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) continue;
                size_t Q = idx(X, Y, Z);
                R sum = uP.c[F.axis] + velT[Q].c[F.axis];
                for (int c = 0; c < 3; ++c) {
                    R t = ds * R(0.25) * velI[Q].c[c] * sum;
                    adv[c] = F.sign > 0 ? adv[c] - t : adv[c] + t;
                }
            }
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                R vis = vis_face(x, y, z, f);
                if (!in_fluid(X, Y, Z)) continue;
                size_t Q = idx(X, Y, Z);
                for (int c = 0; c < 3; ++c) dif[c] += vis * ds / dx * velI[Q].c[c];
            }
            V3<R> r;
            for (int c = 0; c < 3; ++c) r.c[c] = R(1.0) / Dv[P].c[c] * (adv[c] + dif[c] + bv[P].c[c]);
            vel[P] = r;
        });
    }
    // CSComputeVelPredictResidual, FvmColl.compute:3124-3162 (+ host sum and
    // normalisation, FvmSolverGpu.cs:1226-1233).
    double vel_residual() const {
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long long i = 0; i < (long long)N; ++i) {
            R l0 = Dv[i].c[0] * (vel[i].c[0] - velI[i].c[0]);
            R l1 = Dv[i].c[1] * (vel[i].c[1] - velI[i].c[1]);
            R l2 = Dv[i].c[2] * (vel[i].c[2] - velI[i].c[2]);
            s += double(l0 * l0 + l1 * l1 + l2 * l2);
        }
        return std::sqrt(s / (3.0 * double(N)));
    }
    // VelPredict loop, FvmSolverGpu.cs:1238-1282 (fixed count, optional
    // residual break).
    void vel_predict_loop(int n) {
        for (int k = 0; k < n; ++k) {
            vel_sweep();
            if (cf.calc_residual && cf.vel_res_interval > 0 && k % cf.vel_res_interval == 0) {
                res_vel = vel_residual();
                if (res_vel < double(cf.vel_tol)) break;
            }
            std::swap(velI, vel);
        }
        std::swap(velI, vel);
    }

    // ------------------------------------------------ pressure correction
    // CSPresCorrectRhieChowPreCompute, FvmColl.compute:2481-2787
    void op_pres_precompute() {
        if (nonuniform) return nu_pres_precompute();
        const R dx2 = R(2) * dx;
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            R DP = R(0), bP = R(0);
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int a = F.axis;
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z)) {
                    if (!fluid(X, Y, Z)) continue;
                    size_t Q = idx(X, Y, Z);
                    R DInv = R(0.5) * (R(1) / Dv[P].c[a] + R(1) / Dv[Q].c[a]);
                    DP -= (dv / den) * DInv / dx;
                    R fl = R(0.5) * (vel[P].c[a] + vel[Q].c[a]);
                    bP = F.sign > 0 ? bP + fl : bP - fl;
                    // Rhie-Chow: face between low cell L and high cell H.
                    int lx, ly, lz, hx, hy, hz;
                    if (F.sign > 0) { lx = x; ly = y; lz = z; hx = X; hy = Y; hz = Z; }
                    else { lx = X; ly = Y; lz = Z; hx = x; hy = y; hz = z; }
                    const size_t L = idx(lx, ly, lz), H = idx(hx, hy, hz);
                    R presGrad = (p[H] - p[L]) / dx;
                    int HHx = hx + (a == 0), HHy = hy + (a == 1), HHz = hz + (a == 2);
                    int LLx = lx - (a == 0), LLy = ly - (a == 1), LLz = lz - (a == 2);
                    bool hh = in_fluid(HHx, HHy, HHz), ll = in_fluid(LLx, LLy, LLz);
                    // outer cell beyond the face on each side; for the E face
                    // the test pair is (EE, W), for the W face (WW, E).
                    bool outer_far = F.sign > 0 ? hh : ll;   // EE / WW
                    bool outer_near = F.sign > 0 ? ll : hh;  // W  / E
                    R gH = hh ? (p[idx(HHx, HHy, HHz)] - p[L]) / dx2 : (p[H] - p[L]) / dx2;
                    R gL = ll ? (p[H] - p[idx(LLx, LLy, LLz)]) / dx2 : (p[H] - p[L]) / dx2;
                    R ave;
                    if (outer_far || outer_near)
                        ave = R(0.5) * (gH + gL);
                    else
                        ave = presGrad;
                    R vct = -(dv * DInv) / den * (presGrad - ave);
                    bP = F.sign > 0 ? bP + vct : bP - vct;
                } else {
                    int vb = cf.vel_bc[F.bc];
                    if (vb == WF_BND_FIXED_VALUE) {
                        R t = bndv(F.bc, x, y, z).c[a];
                        bP = F.sign > 0 ? bP + t : bP - t;
                    } else if (vb == WF_BND_ZERO_GRAD) {
                        R t = vel[P].c[a];
                        bP = F.sign > 0 ? bP + t : bP - t;
                    }
                    if (cf.pres_bc[F.bc] == WF_BND_FIXED_VALUE) {
                        R DInv = R(1) / Dv[P].c[a];
                        DP -= R(2) * (dv / den) * DInv / dx;
                    }
                }
            }
            Dp[P] = DP;
            bp[P] = bP;
        });
    }
    // CSPresCorrectRhieChow, FvmColl.compute:2790-2848
    void pres_sweep() {
        if (nonuniform) return nu_pres_sweep();
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            R t = R(0);
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) continue;
                size_t Q = idx(X, Y, Z);
                R DInv = R(0.5) * (R(1) / Dv[P].c[F.axis] + R(1) / Dv[Q].c[F.axis]);
                t -= (dv / den) * DInv / dx * pcL[Q];
            }
            pc[P] = (R(1) / Dp[P]) * (t + bp[P]);
        });
    }
    // CSComputePresCorrectResidual, FvmColl.compute:3165-3199 (+ FvmSolverGpu.cs:1354-1362)
    double pres_residual() const {
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (long long i = 0; i < (long long)N; ++i) {
            R l = Dp[i] * (pc[i] - pcL[i]);
            s += double(l * l);
        }
        return std::sqrt(s / double(N));
    }
    // PresCorrect loop, FvmSolverGpu.cs:1372-1415
    void pres_correct_loop(int n) {
        for (int k = 0; k < n; ++k) {
            pres_sweep();
            if (cf.calc_residual && cf.pres_res_interval > 0 && k % cf.pres_res_interval == 0) {
                res_pres = pres_residual();
                if (res_pres < double(cf.pres_tol)) break;
            }
            std::swap(pcL, pc);
        }
        std::swap(pcL, pc);
    }
    // CSApplyPresCorrection, FvmColl.compute:2851-2862
    void op_apply_pres() {
        for_cells([&](int x, int y, int z) {
            size_t P = idx(x, y, z);
            if (flag[P] == WF_CELL_SOLID) return;
            p[P] += pc[P];
        });
    }
    // CSPresNormalization, FvmColl.compute:2865-2880.  The reference reads
    // the reference cell while other groups update it; here the reference
    // value is read once, before any update.
    void op_normalize() {
        R ref = p[idx(2, ny / 2, 2)];
        for_cells([&](int x, int y, int z) {
            size_t P = idx(x, y, z);
            if (flag[P] == WF_CELL_SOLID) return;
            p[P] -= ref;
        });
    }
    bool any_fixed_pres() const {
        for (int f = 0; f < 6; ++f)
            if (cf.pres_bc[f] == WF_BND_FIXED_VALUE) return true;
        return false;
    }
    // CSApplyVelCorrectionDivergenceTheorem, FvmColl.compute:2951-3121
    void op_apply_vel() {
        if (nonuniform) return nu_apply_vel();
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            R pf[6];
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (in_region(X, Y, Z))
                    pf[f] = fluid(X, Y, Z) ? R(0.5) * (pc[P] + pc[idx(X, Y, Z)]) : pc[P];
                else
                    pf[f] = cf.pres_bc[F.bc] == WF_BND_FIXED_VALUE ? R(0) : pc[P];
            }
            V3<R> corr;
            for (int a = 0; a < 3; ++a)
                corr.c[a] = -(dv / den) * (R(1) / Dv[P].c[a]) * (pf[2 * a] - pf[2 * a + 1]) / dx;
            velC[P] = corr;
            for (int a = 0; a < 3; ++a) vel[P].c[a] += corr.c[a];
        });
    }
    // SetPresCorrectFieldtoZero, FvmSolverGpu.cs:1545-1554 (CSSetPresField)
    void op_zero_pres_correct() {
        std::fill(pc.begin(), pc.end(), R(0));
        std::fill(pcL.begin(), pcL.end(), R(0));
    }

    // ---------------------------------------------------------------- PISO
    // CSPisoCalAodUCorrect, PisoColl.compute:71-178
    void piso_aodu() {
        const bool consistent = (cf.compat_flags & WF_COMPAT_PISO_CONSISTENT) != 0;
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            R adv[3] = {R(0), R(0), R(0)}, dif[3] = {R(0), R(0), R(0)};
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) continue;
                size_t Q = idx(X, Y, Z);
                R sum = velT[P].c[F.axis] + velT[Q].c[F.axis];
                for (int c = 0; c < 3; ++c) {
                    R t = ds * R(0.25) * velC[Q].c[c] * sum;
                    adv[c] = F.sign > 0 ? adv[c] + t : adv[c] - t;
                }
            }
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) continue;
                size_t Q = idx(X, Y, Z);
                R vis = consistent ? vis_face(x, y, z, f) : nu;
                for (int c = 0; c < 3; ++c) dif[c] -= vis * ds / dx * velC[Q].c[c];
            }
            aodu[P] = V3<R>{{adv[0] + dif[0], adv[1] + dif[1], adv[2] + dif[2]}};
        });
    }
    // CSPisoPresCorrection, PisoColl.compute:181-256
    void piso_pres_sweep() {
        const bool consistent = (cf.compat_flags & WF_COMPAT_PISO_CONSISTENT) != 0;
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            R coeff = R(0), pt = R(0), vt = R(0);
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                const int a = F.axis;
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                if (!in_fluid(X, Y, Z)) {
                    if (consistent && !in_region(X, Y, Z) && cf.pres_bc[F.bc] == WF_BND_FIXED_VALUE) {
                        R DInv = R(1) / Dv[P].c[a];
                        coeff -= R(2) * (dv / den) * DInv / dx;
                    }
                    continue;
                }
                size_t Q = idx(X, Y, Z);
                R AdInv = R(0.5) * (R(1) / Dv[P].c[a] + R(1) / Dv[Q].c[a]);
                R Aod = R(0.5) * (aodu[P].c[a] + aodu[Q].c[a]);
                if (a == 0) {  // E/W faces parenthesise (AdInv / dx), :205-215
                    coeff -= (dv / den) * (AdInv / dx);
                    pt -= (dv / den) * (AdInv / dx) * pcL[Q];
                } else {
                    coeff -= (dv / den) * AdInv / dx;
                    pt -= (dv / den) * AdInv / dx * pcL[Q];
                }
                vt = F.sign > 0 ? vt - AdInv * Aod : vt + AdInv * Aod;
            }
            pc[P] = (R(1) / coeff) * (pt + vt);
        });
    }
    // CSPisoApplyPresCorrection, PisoColl.compute:259-267
    void piso_apply_pres() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            size_t P = idx(x, y, z);
            p[P] += pc[P];
        });
    }
    // CSPisoVelCorrection, PisoColl.compute:270-337
    void piso_vel() {
        for_cells([&](int x, int y, int z) {
            if (!fluid(x, y, z)) return;
            const size_t P = idx(x, y, z);
            R pf[6];
            for (int f = 0; f < 6; ++f) {
                const Face& F = kFaces[f];
                int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                pf[f] = in_fluid(X, Y, Z) ? R(0.5) * (pc[P] + pc[idx(X, Y, Z)]) : pc[P];
            }
            V3<R> corr;
            for (int a = 0; a < 3; ++a) {
                R grad = (pf[2 * a] - pf[2 * a + 1]) / dx;
                R DInv = R(1) / Dv[P].c[a];
                corr.c[a] = -DInv * (aodu[P].c[a] + dv / den * grad);
            }
            velC[P] = corr;
            for (int a = 0; a < 3; ++a) vel[P].c[a] += corr.c[a];
        });
    }
    // PisoCorrection, FvmSolverGpu.cs:1482-1533
    void op_piso(int n) {
        piso_aodu();
        for (int k = 0; k < n; ++k) {
            piso_pres_sweep();
            std::swap(pcL, pc);
        }
        std::swap(pcL, pc);
        piso_apply_pres();
        piso_vel();
        op_zero_pres_correct();
    }
    // Finished stage, FvmSolverGpu.cs:1103-1118
    void op_end_step() {
        std::swap(velT, vel);
        velI = velT;  // CSCopyVelField, Utils.compute:21-30
        step += 1;
    }

    // Step(), FvmSolverGpu.cs:1050-1121 with fixed iteration counts.
    void full_step() {
        if (les) {
            op_wallfunc();
            op_eddy_vis();
            op_les_term();
        }
        op_vel_precompute();
        vel_predict_loop(cf.vel_iters);
        op_pres_precompute();
        pres_correct_loop(cf.pres_iters);
        op_apply_pres();
        if (!any_fixed_pres()) op_normalize();
        op_apply_vel();
        op_zero_pres_correct();
        if (cf.solver_type == WF_SOLVER_PISO)
            for (int n = 0; n < cf.piso_correctors; ++n) op_piso(cf.pres_iters);
        op_end_step();
    }

    // Sum over fluid cells of |net face flux| of velLastTime (BC-aware, no
    // Rhie-Chow term).
    double mass_imbalance() const {
        double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    if (!fluid(x, y, z)) continue;
                    const size_t P = idx(x, y, z);
                    double div = 0.0;
                    for (int f = 0; f < 6; ++f) {
                        const Face& F = kFaces[f];
                        const int a = F.axis;
                        int X = x + F.ox, Y = y + F.oy, Z = z + F.oz;
                        double uf = 0.0;
                        if (in_region(X, Y, Z)) {
                            if (fluid(X, Y, Z)) uf = 0.5 * (double(velT[P].c[a]) + double(velT[idx(X, Y, Z)].c[a]));
                        } else {
                            int vb = cf.vel_bc[F.bc];
                            if (vb == WF_BND_FIXED_VALUE) uf = double(bndv(F.bc, x, y, z).c[a]);
                            else if (vb == WF_BND_ZERO_GRAD) uf = double(velT[P].c[a]);
                        }
                        div += F.sign * uf;
                    }
                    s += std::fabs(div) * double(ds);
                }
        return s;
    }

    // ---------------------------------------------------------- field access
    std::vector<V3<R>>* vec_field(int f) {
        switch (f) {
            case WF_FIELD_VEL: return &vel;
            case WF_FIELD_VEL_LAST_TIME: return &velT;
            case WF_FIELD_VEL_LAST_ITER: return &velI;
            case WF_FIELD_VEL_CORRECT: return &velC;
            case WF_FIELD_D: return &Dv;
            case WF_FIELD_B: return &bv;
            case WF_FIELD_AODU: return &aodu;
            case WF_FIELD_FACE_EDDY_VIS: return &face;
            default:
                if (f >= WF_FIELD_BND_X0 && f <= WF_FIELD_BND_ZN) return &bnd[f - WF_FIELD_BND_X0];
                return nullptr;
        }
    }
    std::vector<R>* sca_field(int f) {
        switch (f) {
            case WF_FIELD_PRES: return &p;
            case WF_FIELD_PRES_CORRECT: return &pc;
            case WF_FIELD_PRES_CORRECT_LAST_ITER: return &pcL;
            case WF_FIELD_DP: return &Dp;
            case WF_FIELD_BP: return &bp;
            case WF_FIELD_EDDY_VIS: return &eddy;
            case WF_FIELD_DRAG: return &drag;
            default: return nullptr;
        }
    }
};

struct AnyOracle {
    virtual ~AnyOracle() = default;
    virtual int precision() const = 0;
};
template <class R> struct OracleT : AnyOracle {
    Oracle<R> o;
    int precision() const override { return sizeof(R) == 4 ? 32 : 64; }
};

bool valid_config(const wf_config* c) {
    if (!c || c->struct_size != sizeof(wf_config)) return false;
    if (c->nx < 3 || c->ny < 3 || c->nz < 3) return false;
    if (!(c->dx > 0.f) || !(c->dt > 0.f) || !(c->den > 0.f) || !(c->mu >= 0.f)) return false;
    for (int f = 0; f < 6; ++f) {
        if (c->vel_bc[f] < 0 || c->vel_bc[f] > 2) return false;
        if (c->pres_bc[f] < 0 || c->pres_bc[f] > 2) return false;
    }
    if (c->vel_iters < 0 || c->pres_iters < 0 || c->piso_correctors < 0) return false;
    return true;
}

}  // namespace

struct wfo_solver {
    std::unique_ptr<AnyOracle> impl;
};

template <class F> static int dispatch(wfo_solver* h, F&& fn) {
    if (!h || !h->impl) return WF_ERR_INVALID_ARG;
    if (h->impl->precision() == 32) return fn(static_cast<OracleT<float>*>(h->impl.get())->o);
    return fn(static_cast<OracleT<double>*>(h->impl.get())->o);
}
template <class F> static int dispatch_c(const wfo_solver* h, F&& fn) {
    return dispatch(const_cast<wfo_solver*>(h), fn);
}

extern "C" {

int wfo_create(const wf_config* cfg, int precision, int threads, wfo_solver** out) {
    if (!out || !valid_config(cfg) || (precision != 32 && precision != 64)) return WF_ERR_INVALID_ARG;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    auto* h = new (std::nothrow) wfo_solver;
    if (!h) return WF_ERR_OOM;
    try {
        if (precision == 32) {
            auto* o = new OracleT<float>;
            o->o.setup(*cfg);
            h->impl.reset(o);
        } else {
            auto* o = new OracleT<double>;
            o->o.setup(*cfg);
            h->impl.reset(o);
        }
    } catch (...) {
        delete h;
        return WF_ERR_OOM;
    }
    *out = h;
    return WF_OK;
}

int wfo_init_from_background(wfo_solver* h, const wfo_solver* bg, const float pos[3], const float pos_bg[3],
                             float rot_deg) {
    if (!h || !bg || h == bg || !pos || !pos_bg || !h->impl || !bg->impl) return WF_ERR_INVALID_ARG;
    if (h->impl->precision() != bg->impl->precision()) return WF_ERR_INVALID_ARG;
    if (h->impl->precision() == 32) {
        static_cast<OracleT<float>*>(h->impl.get())->o.init_from_background(
            static_cast<const OracleT<float>*>(bg->impl.get())->o, pos, pos_bg, rot_deg);
    } else {
        static_cast<OracleT<double>*>(h->impl.get())->o.init_from_background(
            static_cast<const OracleT<double>*>(bg->impl.get())->o, pos, pos_bg, rot_deg);
    }
    return WF_OK;
}

int wfo_destroy(wfo_solver* h) {
    delete h;
    return WF_OK;
}

int wfo_init_flags(wfo_solver* h, const int32_t* flags, size_t n) {
    return dispatch(h, [&](auto& o) {
        if (!flags || n != o.N) return int(WF_ERR_INVALID_ARG);
        o.init_flags(flags);
        return int(WF_OK);
    });
}
int wfo_init_vel_pres_fields(wfo_solver* h) {
    return dispatch(h, [&](auto& o) { o.init_vel_pres_fields(); return int(WF_OK); });
}
int wfo_set_fixed_value_vel_bnd_cond(wfo_solver* h, float w) {
    return dispatch(h, [&](auto& o) { o.set_fixed_value_vel_bnd_cond(w); return int(WF_OK); });
}
int wfo_set_inflow_plane(wfo_solver* h, const float* pl) {
    return dispatch(h, [&](auto& o) {
        if (!pl) return int(WF_ERR_INVALID_ARG);
        using R = std::decay_t<decltype(o.dx)>;
        for (size_t i = 0; i < o.bnd[0].size(); ++i)
            for (int c = 0; c < 3; ++c) o.bnd[0][i].c[c] = R(pl[i * 3 + c]);
        return int(WF_OK);
    });
}
int wfo_set_face_positions(wfo_solver* h, const float* fx, const float* fy, const float* fz) {
    return dispatch(h, [&](auto& o) {
        using R = std::decay_t<decltype(o.dx)>;
        if (!fx && !fy && !fz) {
            o.nonuniform = false;
            return int(WF_OK);
        }
        if (!fx || !fy || !fz) return int(WF_ERR_INVALID_ARG);
        // the reference has no PISO shader for this grid (FvmSolverGpu.cs:493-496)
        if (o.cf.solver_type != WF_SOLVER_SIMPLE) return int(WF_ERR_UNSUPPORTED);
        const float* f[3] = {fx, fy, fz};
        const int n[3] = {o.nx, o.ny, o.nz};
        for (int a = 0; a < 3; ++a)
            for (int i = 0; i < n[a]; ++i)
                if (!(f[a][i + 1] > f[a][i])) return int(WF_ERR_INVALID_ARG);
        o.fpx.assign(fx, fx + o.nx + 1);
        o.fpy.assign(fy, fy + o.ny + 1);
        o.fpz.assign(fz, fz + o.nz + 1);
        o.flux.assign(size_t(o.nx + 1) * (o.ny + 1) * (o.nz + 1), V3<R>{{R(0), R(0), R(0)}});
        o.nonuniform = true;
        return int(WF_OK);
    });
}
int wfo_get_face_flux(wfo_solver* h, double* out) {
    return dispatch(h, [&](auto& o) {
        if (!out || !o.nonuniform) return int(WF_ERR_INVALID_ARG);
        const size_t m = o.flux.size();
        for (size_t i = 0; i < m; ++i)
            for (int c = 0; c < 3; ++c) out[c * m + i] = double(o.flux[i].c[c]);
        return int(WF_OK);
    });
}
int wfo_step(wfo_solver* h, int n) {
    return dispatch(h, [&](auto& o) {
        if (n < 0) return int(WF_ERR_INVALID_ARG);
        for (int i = 0; i < n; ++i) o.full_step();
        return int(WF_OK);
    });
}

int wfo_field_size(const wfo_solver* h, int field, size_t* points, int* comps) {
    return dispatch_c(h, [&](auto& o) {
        if (!points || !comps) return int(WF_ERR_INVALID_ARG);
        if (auto* v = o.vec_field(field)) { *points = v->size(); *comps = 3; return int(WF_OK); }
        if (auto* s = o.sca_field(field)) { *points = s->size(); *comps = 1; return int(WF_OK); }
        return int(WF_ERR_INVALID_ARG);
    });
}
int wfo_get_field(wfo_solver* h, int field, double* out) {
    return dispatch(h, [&](auto& o) {
        if (!out) return int(WF_ERR_INVALID_ARG);
        if (auto* v = o.vec_field(field)) {
            size_t n = v->size();
            for (int c = 0; c < 3; ++c)
                for (size_t i = 0; i < n; ++i) out[c * n + i] = double((*v)[i].c[c]);
            return int(WF_OK);
        }
        if (auto* s = o.sca_field(field)) {
            for (size_t i = 0; i < s->size(); ++i) out[i] = double((*s)[i]);
            return int(WF_OK);
        }
        return int(WF_ERR_INVALID_ARG);
    });
}
int wfo_set_field(wfo_solver* h, int field, const double* in) {
    return dispatch(h, [&](auto& o) {
        using R = std::decay_t<decltype(o.dx)>;
        if (!in) return int(WF_ERR_INVALID_ARG);
        if (auto* v = o.vec_field(field)) {
            size_t n = v->size();
            for (int c = 0; c < 3; ++c)
                for (size_t i = 0; i < n; ++i) (*v)[i].c[c] = R(in[c * n + i]);
            return int(WF_OK);
        }
        if (auto* s = o.sca_field(field)) {
            for (size_t i = 0; i < s->size(); ++i) (*s)[i] = R(in[i]);
            return int(WF_OK);
        }
        return int(WF_ERR_INVALID_ARG);
    });
}
int wfo_get_flags(wfo_solver* h, int32_t* out) {
    return dispatch(h, [&](auto& o) {
        if (!out) return int(WF_ERR_INVALID_ARG);
        std::copy(o.flag.begin(), o.flag.end(), out);
        return int(WF_OK);
    });
}

#define WFO_OP(name, body) \
    int wfo_op_##name(wfo_solver* h) { return dispatch(h, [&](auto& o) { body; return int(WF_OK); }); }
WFO_OP(wallfunc, o.op_wallfunc())
WFO_OP(eddy_vis, o.op_eddy_vis())
WFO_OP(les_term, o.op_les_term())
WFO_OP(vel_precompute, o.op_vel_precompute())
WFO_OP(pres_precompute, o.op_pres_precompute())
WFO_OP(apply_pres, o.op_apply_pres())
WFO_OP(normalize, o.op_normalize())
WFO_OP(apply_vel, o.op_apply_vel())
WFO_OP(zero_pres_correct, o.op_zero_pres_correct())
WFO_OP(end_step, o.op_end_step())
#undef WFO_OP

int wfo_op_vel_sweeps(wfo_solver* h, int n) {
    return dispatch(h, [&](auto& o) { o.vel_predict_loop(n); return int(WF_OK); });
}
int wfo_op_pres_sweeps(wfo_solver* h, int n) {
    return dispatch(h, [&](auto& o) { o.pres_correct_loop(n); return int(WF_OK); });
}
int wfo_op_piso(wfo_solver* h, int n) {
    return dispatch(h, [&](auto& o) { o.op_piso(n); return int(WF_OK); });
}
int wfo_op_vel_residual(wfo_solver* h, double* out) {
    return dispatch(h, [&](auto& o) {
        if (!out) return int(WF_ERR_INVALID_ARG);
        *out = o.vel_residual();
        return int(WF_OK);
    });
}
int wfo_op_pres_residual(wfo_solver* h, double* out) {
    return dispatch(h, [&](auto& o) {
        if (!out) return int(WF_ERR_INVALID_ARG);
        *out = o.pres_residual();
        return int(WF_OK);
    });
}
int wfo_residuals(wfo_solver* h, double* vel, double* pres) {
    return dispatch(h, [&](auto& o) {
        if (vel) *vel = o.res_vel;
        if (pres) *pres = o.res_pres;
        return int(WF_OK);
    });
}
int wfo_mass_imbalance(wfo_solver* h, double* out) {
    return dispatch(h, [&](auto& o) {
        if (!out) return int(WF_ERR_INVALID_ARG);
        *out = o.mass_imbalance();
        return int(WF_OK);
    });
}

double wfo_log_law_wall_func(double uP, double dx, double nu, double den, int precision) {
    if (precision == 32) return double(Oracle<float>::log_law(float(uP), float(dx), float(nu), float(den)));
    return Oracle<double>::log_law(uP, dx, nu, den);
}

}  // extern "C"
