// Drop-in check of include/cupcfd_gpu/{fvm,benchmark,config}.hpp on the
// reference's real mesh class.
//
// The mesh is built the way a reference run builds it: the JSON
// configuration's "Mesh" block (MeshSourceStructGen, NaivePartitioner) read by
// cupcfd_gpu/config.hpp, then the reference's own
// MeshConfig::buildUnstructuredMesh -> PartitionerNaive ->
// CupCfdSoAMesh<int,double,int>::addData / finalize, compiled unchanged, on P
// ranks of the in-process MPI stand-in (oracle/ref_mpi/mpi.h). On every
// rank's local mesh (owned and ghost cells):
//   1. the GPU mesh's cell->face CSR equals CupCfdSoAMesh::cellFaceMapCSRXAdj
//      and cellFaceMapCSRAdj (CupCfdSoAMesh.cpp:549-668);
//   2. cupcfd::fvm::gpu::GradientPhiGaussDolfyn (nGradient 1 and 2) and
//      FluxMassDolfynFaceLoop return the reference templates' results bit for
//      bit, on the same seeded arrays;
//   3. cupcfd::benchmark::gpu::BenchmarkKernels' GradientPhiGaussDolfyn and
//      FluxMassDolfynFaceLoop benchmarks, on the inputs they generate, return
//      what the reference templates return on those inputs, bit for bit;
//   4. runBenchmark() for each "BenchmarkKernels" entry of the configuration
//      runs its repetitions, every kernel benchmark timed once per repetition.
// Prints "OK realmesh ..." and exits 0 on success.
//
//   realmesh_dropin CONFIG.json RANKS          (needs the GPU)
//   realmesh_dropin --dump DIR CONFIG.json RANKS
//       CPU only: writes each rank's local connectivity (faceCell1, faceCell2,
//       boundary ids, CSR) to DIR/rank<r>.bin for the CPU tests.
//
// Built by `make -C oracle realmesh` where the reference sources exist.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "Communicator.h"
#include "CupCfdSoAMesh.h"
#include "Error.h"
#include "EuclideanVector.h"
#include "GradientKernels.h"
#include "MassKernels.h"
#include "MeshConfig.h"
#include "MeshSourceStructGenConfig.h"
#include "PartitionerNaiveConfig.h"
#include "cupcfd_gpu/benchmark.hpp"
#include "cupcfd_gpu/config.hpp"
#include "cupcfd_gpu/fvm.hpp"

namespace euc = cupcfd::geometry::euclidean;
namespace msh = cupcfd::geometry::mesh;
namespace bgpu = cupcfd::benchmark::gpu;
typedef msh::CupCfdSoAMesh<int, double, int> Mesh;
typedef euc::EuclideanVector<double, 3> Vec;

static int fail(int rank, const char *what) {
    std::printf("FAIL rank %d: %s (%s)\n", rank, what, cupcfd_gpu_last_error());
    return 1;
}

static bool same(const std::vector<double> &a, const std::vector<double> &b) {
    return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), a.size() * sizeof(double)) == 0);
}
static bool same(const std::vector<Vec> &a, const std::vector<Vec> &b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); i++)
        for (int d = 0; d < 3; d++)
            if (std::memcmp(&a[i].cmp[d], &b[i].cmp[d], sizeof(double)) != 0) return false;
    return true;
}

// Builds every rank's mesh from the configuration. The communicators stay
// alive with the meshes (they are never used again after the build).
static int build_meshes(const bgpu::StructGenConfig &sg, int ranks, std::vector<Mesh *> &meshes) {
    if (sg.partitioner != "NaivePartitioner") {
        std::printf("FAIL: the configuration's partitioner is %s; only NaivePartitioner is built here\n",
                    sg.partitioner.c_str());
        return 1;
    }
    meshes.assign((size_t) ranks, nullptr);
    std::vector<int> status((size_t) ranks, 0);
    cupcfd_oracle_mpi::run_ranks(ranks, [&](int r) {
        auto *comm = new cupcfd::comm::Communicator(MPI_COMM_WORLD);
        msh::MeshSourceStructGenConfig<int, double> src(sg.cellX, sg.cellY, sg.cellZ, sg.sMinX, sg.sMaxX, sg.sMinY,
                                                        sg.sMaxY, sg.sMinZ, sg.sMaxZ);
        cupcfd::partitioner::PartitionerNaiveConfig<int, int> part;
        msh::MeshConfig<int, double, int> cfg(part, src);
        Mesh *m = nullptr;
        status[(size_t) r] = (int) cfg.buildUnstructuredMesh(&m, *comm);
        meshes[(size_t) r] = m;
    });
    for (int r = 0; r < ranks; r++)
        if (status[(size_t) r] != CUPCFD_E_SUCCESS || !meshes[(size_t) r]) {
            std::printf("FAIL rank %d: MeshConfig::buildUnstructuredMesh returned %d\n", r, status[(size_t) r]);
            return 1;
        }
    return 0;
}

static void write_ints(std::FILE *f, const std::vector<int32_t> &v) {
    int64_t n = (int64_t) v.size();
    std::fwrite(&n, sizeof n, 1, f);
    if (n) std::fwrite(v.data(), sizeof(int32_t), v.size(), f);
}

static int dump(const std::string &dir, std::vector<Mesh *> &meshes) {
    for (size_t r = 0; r < meshes.size(); r++) {
        Mesh &m = *meshes[r];
        const int nF = m.properties.lFaces, nC = m.properties.lTCells;
        std::vector<int32_t> head = {nC, (int32_t) m.properties.lOCells, nF, (int32_t) m.properties.lBoundaries};
        std::vector<int32_t> c1(nF), c2(nF), bnd(nF);
        for (int f = 0; f < nF; f++) {
            c1[f] = m.getFaceCell1ID(f);
            c2[f] = m.getFaceCell2ID(f);
            bnd[f] = m.getFaceIsBoundary(f) ? m.getFaceBoundaryID(f) : -1;
        }
        std::vector<int32_t> xadj(m.cellFaceMapCSRXAdj.begin(), m.cellFaceMapCSRXAdj.end());
        std::vector<int32_t> adj(m.cellFaceMapCSRAdj.begin(), m.cellFaceMapCSRAdj.end());
        std::string path = dir + "/rank" + std::to_string(r) + ".bin";
        std::FILE *f = std::fopen(path.c_str(), "wb");
        if (!f) return 1;
        for (const auto *v : {&head, &c1, &c2, &bnd, &xadj, &adj}) write_ints(f, *v);
        std::fclose(f);
    }
    std::printf("OK dump %zu ranks\n", meshes.size());
    return 0;
}

// 1 + 2: CSR and the two kernels through the drop-in against the reference
static int check_kernels(int rank, Mesh &mesh, std::default_random_engine &eng) {
    cupcfd_gpu_mesh *gm = nullptr;
    if (cupcfd::fvm::gpu::attach(mesh, &gm) != CUPCFD_E_SUCCESS) return fail(rank, "attach");
    const int nC = mesh.properties.lTCells, nF = mesh.properties.lFaces, nB = mesh.properties.lBoundaries;
    std::vector<int32_t> xadj((size_t) nC + 1), adj(mesh.cellFaceMapCSRAdj.size());
    if (cupcfd_gpu_mesh_get_cell_face_csr(gm, xadj.data(), nC + 1, adj.data(), (int32_t) adj.size()) != CUPCFD_E_SUCCESS)
        return fail(rank, "get_cell_face_csr");
    if (std::vector<int>(xadj.begin(), xadj.end()) != mesh.cellFaceMapCSRXAdj ||
        std::vector<int>(adj.begin(), adj.end()) != mesh.cellFaceMapCSRAdj)
        return fail(rank, "GPU cell->face CSR differs from cellFaceMapCSRXAdj/Adj");

    std::uniform_real_distribution<double> U(-1.0, 1.0);
    auto draw = [&](int n) {
        std::vector<double> v((size_t) n);
        for (double &x : v) x = U(eng);
        return v;
    };
    auto draw_vec = [&](int n) {
        std::vector<Vec> v((size_t) n);
        for (Vec &x : v)
            for (int d = 0; d < 3; d++) x.cmp[d] = U(eng);
        return v;
    };
    for (int ng = 1; ng <= 2; ng++) {
        std::vector<double> phi = draw(nC), phiB = draw(nB);
        std::vector<Vec> g0((size_t) nC), go0((size_t) nC), g1((size_t) nC), go1((size_t) nC);
        auto a = cupcfd::fvm::GradientPhiGaussDolfyn(mesh, ng, phi.data(), nC, phiB.data(), nB, g0.data(), nC,
                                                     go0.data(), nC);
        auto b = cupcfd::fvm::gpu::GradientPhiGaussDolfyn(mesh, ng, phi.data(), nC, phiB.data(), nB, g1.data(), nC,
                                                          go1.data(), nC);
        if ((int) a != CUPCFD_E_SUCCESS || (int) b != CUPCFD_E_SUCCESS) return fail(rank, "gradient status");
        if (!same(g0, g1) || !same(go0, go1)) return fail(rank, "GradientPhiGaussDolfyn differs from the reference");
    }
    {
        std::vector<Vec> du = draw_vec(nC), dv = draw_vec(nC), dw = draw_vec(nC), dp = draw_vec(nC);
        std::vector<double> den = draw(nC), u = draw(nC), v = draw(nC), w = draw(nC), p = draw(nC), ar = draw(nC);
        std::vector<double> denB0 = draw(nB), mf0 = draw(nF), su0 = draw(nC), rf0((size_t) 2 * nF, 0.0);
        std::vector<double> te = draw(nC), ed = draw(nC), vis = draw(nC), t = draw(nC);
        std::vector<double> teB0 = draw(nB), edB0 = draw(nB), visB0 = draw(nB), tB0 = draw(nB);
        std::vector<double> denB1 = denB0, mf1 = mf0, su1 = su0, rf1 = rf0, teB1 = teB0, edB1 = edB0, visB1 = visB0,
                            tB1 = tB0;
        int c0[4] = {0, 0, 0, 0}, c1[4] = {0, 0, 0, 0};
        auto a = cupcfd::fvm::FluxMassDolfynFaceLoop(
            mesh, du.data(), nC, dv.data(), nC, dw.data(), nC, dp.data(), nC, den.data(), nC, denB0.data(), nB,
            u.data(), nC, v.data(), nC, w.data(), nC, mf0.data(), nF, p.data(), nC, ar.data(), nC, su0.data(), nC,
            rf0.data(), 2 * nF, 1e-18, &c0[0], &c0[1], &c0[2], &c0[3], true, true, true, true, te.data(), nC,
            teB0.data(), nB, ed.data(), nC, edB0.data(), nB, vis.data(), nC, visB0.data(), nB, t.data(), nC,
            tB0.data(), nB);
        auto b = cupcfd::fvm::gpu::FluxMassDolfynFaceLoop(
            mesh, du.data(), nC, dv.data(), nC, dw.data(), nC, dp.data(), nC, den.data(), nC, denB1.data(), nB,
            u.data(), nC, v.data(), nC, w.data(), nC, mf1.data(), nF, p.data(), nC, ar.data(), nC, su1.data(), nC,
            rf1.data(), 2 * nF, 1e-18, &c1[0], &c1[1], &c1[2], &c1[3], true, true, true, true, te.data(), nC,
            teB1.data(), nB, ed.data(), nC, edB1.data(), nB, vis.data(), nC, visB1.data(), nB, t.data(), nC,
            tB1.data(), nB);
        if ((int) a != CUPCFD_E_SUCCESS || (int) b != CUPCFD_E_SUCCESS) return fail(rank, "mass flux status");
        if (!same(mf0, mf1) || !same(rf0, rf1) || !same(su0, su1) || !same(denB0, denB1) || !same(teB0, teB1) ||
            !same(edB0, edB1) || !same(visB0, visB1) || !same(tB0, tB1) || std::memcmp(c0, c1, sizeof c0) != 0)
            return fail(rank, "FluxMassDolfynFaceLoop differs from the reference");
    }
    return 0;
}

// 3 + 4: the benchmark entry points
static int check_benchmarks(int rank, Mesh &mesh, const std::vector<bgpu::KernelBenchmarkConfig> &cfgs) {
    std::shared_ptr<Mesh> ptr(&mesh, [](Mesh *) {});
    bgpu::BenchmarkKernels<Mesh, Vec> bk("KernelCheck", ptr, 1, 1000u + (unsigned) rank);
    bk.keepLastCalls(true);
    if ((int) bk.GradientPhiGaussDolfynBenchmark() != CUPCFD_E_SUCCESS) return fail(rank, "gradient benchmark");
    if ((int) bk.FluxMassDolfynFaceLoopBenchmark() != CUPCFD_E_SUCCESS) return fail(rank, "mass benchmark");
    {
        auto c = bk.lastGradientInputs();
        const int nC = mesh.properties.lTCells, nB = mesh.properties.lBoundaries;
        auto rc = cupcfd::fvm::GradientPhiGaussDolfyn(mesh, c.nGradient, c.phiCell.data(), nC, c.phiBoundary.data(), nB,
                                                      c.dPhidxCell.data(), nC, c.dPhidxoCell.data(), nC);
        const auto &g = bk.lastGradientResults();
        if ((int) rc != CUPCFD_E_SUCCESS || !same(c.dPhidxCell, g.dPhidxCell) || !same(c.dPhidxoCell, g.dPhidxoCell))
            return fail(rank, "GradientPhiGaussDolfynBenchmark differs from the reference on its inputs");
    }
    {
        auto c = bk.lastMassInputs();
        const int nC = mesh.properties.lTCells, nB = mesh.properties.lBoundaries, nF = mesh.properties.lFaces;
        auto rc = cupcfd::fvm::FluxMassDolfynFaceLoop(
            mesh, c.dudx.data(), nC, c.dvdx.data(), nC, c.dwdx.data(), nC, c.dpdx.data(), nC, c.denCell.data(), nC,
            c.denBoundary.data(), nB, c.uCell.data(), nC, c.vCell.data(), nC, c.wCell.data(), nC, c.massFlux.data(),
            nF, c.p.data(), nC, c.ar.data(), nC, c.su.data(), nC, c.rface.data(), 2 * nF, c.small, &c.icinl, &c.icout,
            &c.icsym, &c.icwal, c.solveTurbEnergy, c.solveTurbDiss, c.solveVisc, c.solveEnthalpy, c.teCell.data(), nC,
            c.teBoundary.data(), nB, c.edCell.data(), nC, c.edBoundary.data(), nB, c.viseffCell.data(), nC,
            c.viseffBoundary.data(), nB, c.tCell.data(), nC, c.tBoundary.data(), nB);
        const auto &o = bk.lastMassResults();
        if ((int) rc != CUPCFD_E_SUCCESS || !same(c.massFlux, o.massFlux) || !same(c.rface, o.rface) ||
            !same(c.su, o.su) || !same(c.denBoundary, o.denBoundary) || !same(c.viseffBoundary, o.viseffBoundary) ||
            c.icinl != o.icinl || c.icout != o.icout || c.icsym != o.icsym || c.icwal != o.icwal)
            return fail(rank, "FluxMassDolfynFaceLoopBenchmark differs from the reference on its inputs");
    }
    for (const auto &cfg : cfgs) {
        bgpu::BenchmarkKernels<Mesh, Vec> run(cfg, ptr);
        if ((int) run.runBenchmark() != CUPCFD_E_SUCCESS) return fail(rank, "runBenchmark");
        const size_t perRep = 11;  // kernel benchmarks of one repetition
        if (run.timings().size() != perRep * (size_t) cfg.repetitions) return fail(rank, "runBenchmark timings");
        double tg = 0;
        for (const auto &t : run.timings())
            if (t.name == "GradientPhiGaussDolfynBenchmark") tg += t.seconds;
        if (rank == 0)
            std::printf("benchmark %s: %ld repetitions, GradientPhiGaussDolfynBenchmark %.3f ms per call on %ld cells\n",
                        cfg.benchmarkName.c_str(), cfg.repetitions, 1e3 * tg / (double) cfg.repetitions,
                        run.timings().front().localCells);
    }
    return 0;
}

int main(int argc, char **argv) {
    bool dumpMode = argc > 1 && std::strcmp(argv[1], "--dump") == 0;
    if ((dumpMode && argc < 5) || (!dumpMode && argc < 3)) {
        std::printf("usage: %s CONFIG.json RANKS | --dump DIR CONFIG.json RANKS\n", argv[0]);
        return 2;
    }
    const char *cfgPath = argv[dumpMode ? 3 : 1];
    const int ranks = std::atoi(argv[dumpMode ? 4 : 2]);
    bgpu::Json root;
    if (bgpu::read_json(cfgPath, root) != CUPCFD_E_SUCCESS) return fail(-1, "configuration unreadable");
    bgpu::StructGenConfig sg;
    if (bgpu::structgen_mesh(root, sg) != CUPCFD_E_SUCCESS) return fail(-1, "no MeshSourceStructGen mesh");
    std::vector<bgpu::KernelBenchmarkConfig> cfgs;
    if (bgpu::kernel_benchmarks(root, cfgs) != CUPCFD_E_SUCCESS) return fail(-1, "no kernel benchmarks");
    std::vector<Mesh *> meshes;
    if (build_meshes(sg, ranks, meshes)) return 1;
    if (dumpMode) return dump(argv[2], meshes);
    std::default_random_engine eng(7);
    long cells = 0;
    for (int r = 0; r < ranks; r++) {
        Mesh &m = *meshes[(size_t) r];
        if (check_kernels(r, m, eng) || check_benchmarks(r, m, cfgs)) return 1;
        cells += m.properties.lTCells;
        cupcfd::fvm::gpu::release(m);
    }
    std::printf("OK realmesh %dx%dx%d on %d ranks (%ld local cells): CSR, GradientPhiGaussDolfyn, "
                "FluxMassDolfynFaceLoop and the kernel benchmarks bit-identical to the reference\n",
                sg.cellX, sg.cellY, sg.cellZ, ranks, cells);
    return 0;
}
