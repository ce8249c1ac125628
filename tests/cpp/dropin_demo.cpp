// Drop-in check of include/cupcfd_gpu/fvm.hpp against the reference itself.
//
// Builds a structured mesh with the reference's MeshStructGenSource, lays it
// out as a one-rank mesh behind the getter interface the reference kernels
// use, then calls, with the SAME argument lists and the reference's own
// EuclideanVector<double,3> arrays:
//   cupcfd::fvm::GradientPhiGaussDolfyn        (reference CPU template)
//   cupcfd::fvm::gpu::GradientPhiGaussDolfyn   (this library, B200)
// and likewise FluxMassDolfynFaceLoop with inlet/outlet/symmetry/wall
// regions, the mass boundary / region loops and the momentum loops
// (FluxUVWDolfynFaceLoop1, RegionLoop1, BndsLoop1), and requires
// bit-identical results. Exit status 0 on success.
//
// Built by `make -C oracle dropin` (needs the reference sources); the binary
// lands in oracle/_ref/ next to the reference build it links.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "Error.h"
#include "EuclideanVector.h"
#include "GradientKernels.h"
#include "MassKernels.h"
#include "MeshStructGenSource.h"
#include "UVWKernels.h"
#include "cupcfd_gpu/fvm.hpp"

namespace euc = cupcfd::geometry::euclidean;
namespace msh = cupcfd::geometry::mesh;
typedef msh::UnstructuredMeshInterface<int, int, double, int> Mesh;

static int fail(const char *what) {
    std::printf("FAIL: %s (%s)\n", what, cupcfd_gpu_last_error());
    return 1;
}

static bool same(const std::vector<euc::EuclideanVector<double, 3>> &a, const std::vector<euc::EuclideanVector<double, 3>> &b) {
    for (size_t i = 0; i < a.size(); i++)
        for (int d = 0; d < 3; d++)
            if (!(a[i].cmp[d] == b[i].cmp[d])) return false;
    return true;
}

// FluxMassDolfynBoundaryLoop1, 3, 4, 2, RegionLoop, 5 in a solver step's
// order through the reference's templates and through the drop-in, on the
// same mesh (real type T) and inputs: nullptr when every scalar and array is
// bit-identical, else what differs.
template <class T>
static bool same_bits(const std::vector<T> &a, const std::vector<T> &b) {
    return a.size() == b.size() && std::memcmp(a.data(), b.data(), sizeof(T) * a.size()) == 0;
}
template <class T>
static bool same_bits(T a, T b) { return std::memcmp(&a, &b, sizeof(T)) == 0; }

template <class T, class M, class R>
static const char *boundary_chain(M &mesh, int nC, int nF, int nB, int nR, R &rng) {
    namespace ref = cupcfd::fvm;
    namespace g = cupcfd::fvm::gpu;
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::vector<T> mf0(nF);
    for (auto &x : mf0) x = (T) (U(rng) * 1e-2);
    T fin[2], rate[2], fo4[2], fo2[2], fo5[2] = {(T) 0.125, (T) 0.125};
    std::vector<T> mf[2] = {mf0, mf0}, ub[2], vb[2], wb[2], fr[2], ff[2], s5[2];
    std::vector<T> denb(nB);
    for (auto &x : denb) x = (T) (1.0 + 0.1 * U(rng));
    for (int r = 0; r < 2; r++) {
        ub[r].assign(nB, (T) 0.01); vb[r].assign(nB, (T) 0.02); wb[r].assign(nB, (T) 0.03);
        fr[r].assign(nR, (T) 0.001); ff[r].assign(nR, (T) -1.0); s5[r].assign(nC, (T) 0.5);
    }
    cupcfd::error::eCodes st[2][6];
    st[0][0] = ref::FluxMassDolfynBoundaryLoop1(mesh, mf[0].data(), nF, &fin[0]);
    st[1][0] = g::FluxMassDolfynBoundaryLoop1(mesh, mf[1].data(), nF, &fin[1]);
    st[0][1] = ref::FluxMassDolfynBoundaryLoop3(mesh, fin[0], &rate[0]);
    st[1][1] = g::FluxMassDolfynBoundaryLoop3(mesh, fin[1], &rate[1]);
    st[0][2] = ref::FluxMassDolfynBoundaryLoop4(mesh, mf[0].data(), nF, ub[0].data(), nB, vb[0].data(), nB,
                                                wb[0].data(), nB, denb.data(), nB, rate[0], &fo4[0]);
    st[1][2] = g::FluxMassDolfynBoundaryLoop4(mesh, mf[1].data(), nF, ub[1].data(), nB, vb[1].data(), nB,
                                              wb[1].data(), nB, denb.data(), nB, rate[1], &fo4[1]);
    st[0][3] = ref::FluxMassDolfynBoundaryLoop2(mesh, mf[0].data(), nF, fr[0].data(), nR, &fo2[0]);
    st[1][3] = g::FluxMassDolfynBoundaryLoop2(mesh, mf[1].data(), nF, fr[1].data(), nR, &fo2[1]);
    st[0][4] = ref::FluxMassDolfynRegionLoop(mesh, ff[0].data(), nR, fr[0].data(), nR, fin[0]);
    st[1][4] = g::FluxMassDolfynRegionLoop(mesh, ff[1].data(), nR, fr[1].data(), nR, fin[1]);
    st[0][5] = ref::FluxMassDolfynBoundaryLoop5(mesh, mf[0].data(), nF, s5[0].data(), nC, ub[0].data(), nB,
                                                vb[0].data(), nB, wb[0].data(), nB, (T) 1.25, true, false, true,
                                                ff[0].data(), nR, &fo5[0]);
    st[1][5] = g::FluxMassDolfynBoundaryLoop5(mesh, mf[1].data(), nF, s5[1].data(), nC, ub[1].data(), nB,
                                              vb[1].data(), nB, wb[1].data(), nB, (T) 1.25, true, false, true,
                                              ff[1].data(), nR, &fo5[1]);
    for (int k = 0; k < 6; k++)
        if (st[0][k] != cupcfd::error::E_SUCCESS || st[1][k] != cupcfd::error::E_SUCCESS)
            return "boundary loop status";
    if (!(same_bits(fin[0], fin[1]) && same_bits(rate[0], rate[1]) && same_bits(fo4[0], fo4[1]) &&
          same_bits(fo2[0], fo2[1]) && same_bits(fo5[0], fo5[1])))
        return "boundary loop scalars differ from the reference";
    if (!(same_bits(mf[0], mf[1]) && same_bits(ub[0], ub[1]) && same_bits(vb[0], vb[1]) && same_bits(wb[0], wb[1]) &&
          same_bits(fr[0], fr[1]) && same_bits(ff[0], ff[1]) && same_bits(s5[0], s5[1])))
        return "boundary loop arrays differ from the reference";
    return nullptr;
}

int main(int argc, char **argv) {
    int n = argc > 1 ? std::atoi(argv[1]) : 12;
    int nx = n, ny = n - 1, nz = n + 2;
    msh::MeshStructGenSource<int, double> src(nx, ny, nz, 0.0, 1.0, -1.0, 1.0, 0.0, 2.0);
    int nC, nF, nB, nV;
    src.getCellCount(&nC);
    src.getFaceCount(&nF);
    src.getBoundaryCount(&nB);
    src.getVertexCount(&nV);
    std::vector<int> fl(nF), cl(nC), c1(nF), c2(nF, -1), bnd(nF, -1);
    for (int i = 0; i < nF; i++) fl[i] = i;
    for (int i = 0; i < nC; i++) cl[i] = i;
    std::vector<char> isB(nF);
    src.getFaceIsBoundary((bool *) isB.data(), nF, fl.data(), nF);
    src.getFaceCell1Labels(c1.data(), nF, fl.data(), nF);
    std::vector<int> inner, outer;
    for (int f = 0; f < nF; f++) (isB[f] ? outer : inner).push_back(f);
    std::vector<int> tmp(inner.size()), bl(outer.size());
    src.getFaceCell2Labels(tmp.data(), (int) inner.size(), inner.data(), (int) inner.size());
    for (size_t k = 0; k < inner.size(); k++) c2[inner[k]] = tmp[k];
    src.getFaceBoundaryLabels(bl.data(), (int) outer.size(), outer.data(), (int) outer.size());
    for (size_t k = 0; k < outer.size(); k++) bnd[outer[k]] = bl[k];
    std::vector<double> lam(nF), area(nF), vol(nC);
    src.getFaceLambda(lam.data(), nF, fl.data(), nF);
    src.getFaceArea(area.data(), nF, fl.data(), nF);
    src.getCellVolume(vol.data(), nC, cl.data(), nC);
    std::vector<euc::EuclideanVector<double, 3>> nrm(nF);
    std::vector<euc::EuclideanPoint<double, 3>> fc(nF), cc(nC);
    src.getFaceNormal(nrm.data(), nF, fl.data(), nF);
    src.getFaceCenter(fc.data(), nF, fl.data(), nF);
    src.getCellCenter(cc.data(), nC, cl.data(), nC);
    std::vector<double> S(3 * nF), X(3 * nF), C(3 * nC), Z(3 * nF, 0.0);
    for (int f = 0; f < nF; f++)
        for (int d = 0; d < 3; d++) { S[3 * f + d] = nrm[f].cmp[d]; X[3 * f + d] = fc[f].cmp[d]; }
    for (int c = 0; c < nC; c++)
        for (int d = 0; d < 3; d++) C[3 * c + d] = cc[c].cmp[d];
    // four boundary regions: inlet, outlet, symmetry, wall
    int nR = 4;
    std::vector<int> rtype = {msh::RTYPE_INLET, msh::RTYPE_OUTLET, msh::RTYPE_SYMP, msh::RTYPE_WALL}, breg(nB);
    std::vector<double> ruvw = {1.0, 0.5, -0.25, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0}, rden = {1.2, 1, 1, 1};
    for (int b = 0; b < nB; b++) breg[b] = b % nR;

    Mesh mesh;
    mesh.properties = {nC, 0, nC, nF, nB, nR};
    mesh.a = {c1.data(), c2.data(), bnd.data(), lam.data(), S.data(), X.data(), area.data(), Z.data(), Z.data(),
              C.data(), vol.data(), breg.data(), rtype.data(), ruvw.data(), rden.data()};
    std::vector<int> bface(nB);  // getBoundaryFaceID
    for (int f = 0; f < nF; f++)
        if (bnd[f] > -1) bface[bnd[f]] = f;
    std::vector<double> splvl = {0.5, 0.75, 0.25, 1.0};  // getRegionSplvl
    mesh.a.boundaryFace = bface.data();
    mesh.a.regionSplvl = splvl.data();
    // momentum-loop geometry and state (getFaceRLencos, getBoundaryDistance,
    // boundary shear, region force tangents), set before the first attach
    std::vector<double> rlc(nF), bdist(nB), shear(3 * nB, 0.0), ftan(3 * nR, 0.0);
    {
        std::mt19937_64 g(7);
        std::uniform_real_distribution<double> u01(0.0, 1.0);
        for (auto &x : rlc) x = 0.25 + u01(g);
        for (auto &x : bdist) x = 0.01 + 0.1 * u01(g);
    }
    mesh.a.faceRLencos = rlc.data();
    mesh.a.boundaryDistance = bdist.data();
    mesh.a.boundaryShear = shear.data();
    mesh.a.regionForceTangent = ftan.data();

    std::mt19937_64 rng(20261203);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    std::normal_distribution<double> N01(0.0, 1.0);
    std::vector<double> phi(nC), phiB(nB);
    for (auto &x : phi) x = U(rng);
    for (auto &x : phiB) x = U(rng);

    // ---- GradientPhiGaussDolfyn: identical call sites, two namespaces
    for (int nGrad = 1; nGrad <= 3; nGrad++) {
        std::vector<euc::EuclideanVector<double, 3>> g1(nC), go1(nC), g2(nC), go2(nC);
        cupcfd::error::eCodes s1 = cupcfd::fvm::GradientPhiGaussDolfyn(mesh, nGrad, phi.data(), nC, phiB.data(), nB,
                                                                        g1.data(), nC, go1.data(), nC);
        cupcfd::error::eCodes s2 = cupcfd::fvm::gpu::GradientPhiGaussDolfyn(mesh, nGrad, phi.data(), nC, phiB.data(), nB,
                                                                             g2.data(), nC, go2.data(), nC);
        if (s1 != cupcfd::error::E_SUCCESS || s2 != cupcfd::error::E_SUCCESS) return fail("gradient status");
        if (!same(g1, g2) || !same(go1, go2)) return fail("gradient differs from the reference");
    }

    // ---- FluxMassDolfynFaceLoop with all region types
    std::vector<euc::EuclideanVector<double, 3>> du(nC), dv(nC), dw(nC), dp(nC);
    for (int c = 0; c < nC; c++)
        for (int d = 0; d < 3; d++) { du[c].cmp[d] = N01(rng); dv[c].cmp[d] = N01(rng); dw[c].cmp[d] = N01(rng); dp[c].cmp[d] = N01(rng); }
    std::vector<double> den(nC), u(nC), v(nC), w(nC), p(nC), ar(nC), te(nC), ed(nC), vis(nC), t(nC);
    for (int c = 0; c < nC; c++) {
        den[c] = 0.9 + 0.2 * (U(rng) + 1) / 2; u[c] = N01(rng); v[c] = N01(rng); w[c] = N01(rng);
        p[c] = U(rng); ar[c] = 0.9 + 0.2 * (U(rng) + 1) / 2; te[c] = U(rng); ed[c] = U(rng); vis[c] = U(rng); t[c] = U(rng);
    }
    struct Out {
        std::vector<double> mf, su, rf, denB, teB, edB, visB, tB;
        int c[4];
    } o[2];
    for (int r = 0; r < 2; r++) {
        o[r].mf.assign(nF, 0.125); o[r].su.assign(nC, 0.5); o[r].rf.assign(2 * nF, -3.0); o[r].denB.assign(nB, 0.0);
        o[r].teB.assign(nB, 0.0); o[r].edB.assign(nB, 0.0); o[r].visB.assign(nB, 0.0); o[r].tB.assign(nB, 0.0);
        o[r].c[0] = 1; o[r].c[1] = o[r].c[2] = o[r].c[3] = 0;
    }
#define MASS_ARGS(O)                                                                                                  \
    mesh, du.data(), nC, dv.data(), nC, dw.data(), nC, dp.data(), nC, den.data(), nC, O.denB.data(), nB, u.data(), nC, \
        v.data(), nC, w.data(), nC, O.mf.data(), nF, p.data(), nC, ar.data(), nC, O.su.data(), nC, O.rf.data(), 2 * nF,  \
        1e-18, &O.c[0], &O.c[1], &O.c[2], &O.c[3], true, true, true, true, te.data(), nC, O.teB.data(), nB, ed.data(),  \
        nC, O.edB.data(), nB, vis.data(), nC, O.visB.data(), nB, t.data(), nC, O.tB.data(), nB
    cupcfd::error::eCodes m1 = cupcfd::fvm::FluxMassDolfynFaceLoop(MASS_ARGS(o[0]));
    cupcfd::error::eCodes m2 = cupcfd::fvm::gpu::FluxMassDolfynFaceLoop(MASS_ARGS(o[1]));
    if (m1 != cupcfd::error::E_SUCCESS || m2 != cupcfd::error::E_SUCCESS) return fail("mass flux status");
    if (o[0].mf != o[1].mf || o[0].su != o[1].su || o[0].rf != o[1].rf || o[0].denB != o[1].denB ||
        o[0].teB != o[1].teB || o[0].edB != o[1].edB || o[0].visB != o[1].visB || o[0].tB != o[1].tB)
        return fail("mass flux differs from the reference");
    for (int k = 0; k < 4; k++)
        if (o[0].c[k] != o[1].c[k]) return fail("region counters differ");

    // ---- FluxMassDolfynBoundaryLoop1-5 and FluxMassDolfynRegionLoop (outlet region 1, inlet region 0)
    if (const char *e = boundary_chain<double>(mesh, nC, nF, nB, nR, rng)) return fail(e);
    // ---- FluxUVWDolfynFaceLoop1, RegionLoop1, BndsLoop1 (boundary 0, on face 0, is an inlet)
    {
        namespace ref = cupcfd::fvm;
        namespace g = cupcfd::fvm::gpu;
        std::uniform_real_distribution<double> Usm(1e-6, 1e-2);
        auto draw = [&](int n) { std::vector<double> a(n); for (auto &x : a) x = Usm(rng); return a; };
        std::vector<double> uc = draw(nC), vc = draw(nC), wc = draw(nC), visc = draw(nC), visb = draw(nB);
        std::vector<double> mf0 = draw(nF);
        for (int f = 0; f < nF; f += 3) mf0[f] = -mf0[f];
        std::vector<euc::EuclideanVector<double, 3>> du(nC), dv(nC), dw(nC);
        for (int c = 0; c < nC; c++)
            for (int d = 0; d < 3; d++) { du[c].cmp[d] = 1e-2 * N01(rng); dv[c].cmp[d] = 1e-2 * N01(rng); dw[c].cmp[d] = 1e-2 * N01(rng); }
        std::vector<double> mf[2] = {mf0, mf0}, rf[2], ub[2], vb[2], wb[2], s[2][6];
        std::vector<double> rf0(2 * nF);
        for (auto &x : rf0) x = U(rng);
        std::vector<double> sa0 = draw(nC), ub0 = draw(nB);
        for (int r = 0; r < 2; r++) {
            rf[r] = rf0; ub[r] = ub0; vb[r] = ub0; wb[r] = ub0;
            for (int q = 0; q < 6; q++) s[r][q] = sa0;
        }
        cupcfd::error::eCodes st0 = ref::FluxUVWDolfynFaceLoop1(
            mesh, 0.9, 1e-18, uc.data(), nC, vc.data(), nC, wc.data(), nC, ub[0].data(), nB, vb[0].data(), nB,
            wb[0].data(), nB, visc.data(), nC, visb.data(), nB, mf[0].data(), nF, du.data(), nC, dv.data(), nC, dw.data(),
            nC, rf[0].data(), 2 * nF, s[0][0].data(), nC, s[0][1].data(), nC, s[0][2].data(), nC, s[0][3].data(), nC,
            s[0][4].data(), nC, s[0][5].data(), nC);
        std::vector<double> shearRef = shear;
        std::fill(shear.begin(), shear.end(), 0.0);
        cupcfd::error::eCodes st1 = g::FluxUVWDolfynFaceLoop1(
            mesh, 0.9, 1e-18, uc.data(), nC, vc.data(), nC, wc.data(), nC, ub[1].data(), nB, vb[1].data(), nB,
            wb[1].data(), nB, visc.data(), nC, visb.data(), nB, mf[1].data(), nF, du.data(), nC, dv.data(), nC, dw.data(),
            nC, rf[1].data(), 2 * nF, s[1][0].data(), nC, s[1][1].data(), nC, s[1][2].data(), nC, s[1][3].data(), nC,
            s[1][4].data(), nC, s[1][5].data(), nC);
        if (st0 != cupcfd::error::E_SUCCESS || st1 != cupcfd::error::E_SUCCESS) return fail("momentum loop status");
        if (mf[0] != mf[1] || rf[0] != rf[1] || ub[0] != ub[1] || vb[0] != vb[1] || wb[0] != wb[1] || shear != shearRef)
            return fail("momentum loop face / boundary arrays differ from the reference");
        for (int q = 0; q < 6; q++)
            if (s[0][q] != s[1][q]) return fail("momentum loop su..aw differ from the reference");
        std::fill(ftan.begin(), ftan.end(), 7.0);
        ref::FluxUVWDolfynRegionLoop1(mesh);
        ref::FluxUVWDolfynBndsLoop1(mesh);
        std::vector<double> ftRef = ftan;
        std::fill(ftan.begin(), ftan.end(), 7.0);
        if (g::FluxUVWDolfynRegionLoop1(mesh) != cupcfd::error::E_SUCCESS ||
            g::FluxUVWDolfynBndsLoop1(mesh) != cupcfd::error::E_SUCCESS)
            return fail("momentum region / boundary loop status");
        if (ftan != ftRef) return fail("region force tangents differ from the reference");
    }
    cupcfd::fvm::gpu::release(mesh);

    // ---- GradientPhiGaussDolfyn on a T = float mesh (the same geometry
    // rounded to float): the reference's float instantiation and the drop-in
    typedef msh::UnstructuredMeshInterface<int, int, float, int> MeshF;
    auto tof = [](const std::vector<double> &v) { return std::vector<float>(v.begin(), v.end()); };
    std::vector<float> lamF = tof(lam), SF = tof(S), XF = tof(X), areaF = tof(area), ZF = tof(Z), CF = tof(C),
                       volF = tof(vol), ruvwF = tof(ruvw), rdenF = tof(rden), phiF = tof(phi), phiBF = tof(phiB);
    MeshF meshF;
    meshF.properties = {nC, 0, nC, nF, nB, nR};
    meshF.a = {c1.data(), c2.data(), bnd.data(), lamF.data(), SF.data(), XF.data(), areaF.data(), ZF.data(), ZF.data(),
               CF.data(), volF.data(), breg.data(), rtype.data(), ruvwF.data(), rdenF.data()};
    meshF.a.boundaryFace = bface.data();
    std::vector<float> splvlF = tof(splvl), rlcF = tof(rlc), bdistF = tof(bdist), shearF(3 * nB, 0.f), ftanF(3 * nR, 0.f);
    meshF.a.regionSplvl = splvlF.data();
    meshF.a.faceRLencos = rlcF.data();
    meshF.a.boundaryDistance = bdistF.data();
    meshF.a.boundaryShear = shearF.data();
    meshF.a.regionForceTangent = ftanF.data();
    for (int nGrad = 1; nGrad <= 3; nGrad++) {
        std::vector<euc::EuclideanVector<float, 3>> g1(nC), go1(nC), g2(nC), go2(nC);
        cupcfd::error::eCodes s1 = cupcfd::fvm::GradientPhiGaussDolfyn(meshF, nGrad, phiF.data(), nC, phiBF.data(), nB,
                                                                        g1.data(), nC, go1.data(), nC);
        cupcfd::error::eCodes s2 = cupcfd::fvm::gpu::GradientPhiGaussDolfyn(meshF, nGrad, phiF.data(), nC, phiBF.data(),
                                                                             nB, g2.data(), nC, go2.data(), nC);
        if (s1 != cupcfd::error::E_SUCCESS || s2 != cupcfd::error::E_SUCCESS) return fail("float gradient status");
        for (int i = 0; i < nC; i++)
            for (int d = 0; d < 3; d++)
                if (std::memcmp(&g1[i].cmp[d], &g2[i].cmp[d], 4) != 0 || std::memcmp(&go1[i].cmp[d], &go2[i].cmp[d], 4) != 0)
                    return fail("float gradient differs from the reference's float instantiation");
    }
    // ---- the boundary / region loops on the float mesh
    if (const char *e = boundary_chain<float>(meshF, nC, nF, nB, nR, rng)) return fail(e);
    cupcfd::fvm::gpu::release(meshF);
    std::printf("OK dropin %dx%dx%d: %d cells, %d faces; gradient (nGradient 1-3, double and float meshes), mass "
                "flux, the boundary / region loops (double and float meshes) and the momentum loops "
                "bit-identical\n", nx, ny, nz, nC, nF);
    return 0;
}
