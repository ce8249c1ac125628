// cupcfd_gpu/benchmark.hpp - the reference's kernel benchmark entry points
// (cupcfd::benchmark::BenchmarkKernels, src/benchmarks/implementation/
// component/BenchmarkKernels.cpp) run through the B200 drop-in of
// cupcfd_gpu/fvm.hpp, in namespace cupcfd::benchmark::gpu.
//
// Same entry points by name: runBenchmark() (BenchmarkKernels.cpp:55-115)
// repeats, `repetitions` times and in the reference's order, the kernel
// benchmarks this library provides:
//   GradientPhiGaussDolfynBenchmark        (:118-194)
//   FluxMassDolfynFaceLoopBenchmark        (:197-326)
//   FluxMassDolfynBoundaryLoop1-5Benchmark, FluxMassDolfynRegionLoopBenchmark
//   FluxUVWDolfynFaceLoop1Benchmark, FluxUVWDolfynRegionLoop1Benchmark,
//   FluxUVWDolfynBndsLoop1Benchmark
// The reference's FluxScalarDolfynFaceLoop and viscosity benchmarks have no
// kernels in this library and are not run.
//
// Each benchmark allocates its arrays as the reference does, fills them from
// U[1e-6, 1e-2] (randomUniform, ArrayKernels.ipp:307-315), and times the
// kernel call alone. Differences from the reference, all on purpose:
//   - the generator is std::default_random_engine seeded once per benchmark
//     object with `seed`, not from std::random_device per array, so a run can
//     be repeated and checked;
//   - arrays the reference leaves uninitialised (the gradients and the
//     te/ed/viseff/t arrays of FluxMassDolfynFaceLoop, flowFact of boundary
//     loop 5, the velocity gradients of FluxUVWDolfynFaceLoop1) are drawn
//     from the same distribution;
//   - the timer is std::chrono::steady_clock around the call (the drop-in
//     returns once the results are in the caller's arrays), recorded per
//     call in timings() with the sizes the reference's TreeTimer logs
//     (TreeTimer is not part of this library).
// With keepLastCalls(true) the inputs and results of the latest
// GradientPhiGaussDolfyn and FluxMassDolfynFaceLoop calls are kept, so the
// same inputs can be given to another implementation and compared.
//
// Mesh: the mesh type the reference benchmark holds (a CupCfdSoAMesh, or the
// UnstructuredMeshInterface<M,I,T,L> it derives from); Vec: its vector type
// (cupcfd::geometry::euclidean::EuclideanVector<T,3>), or any type with
// a `T cmp[3]` member.
#pragma once

#include <chrono>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "cupcfd_gpu/config.hpp"
#include "cupcfd_gpu/fvm.hpp"

namespace cupcfd {
namespace benchmark {
namespace gpu {

using cupcfd::fvm::gpu::ecode_t;

// One timed kernel call.
struct Timing {
    std::string name;  // the reference's timer block name, e.g. "GradientPhiGaussDolfynBenchmark"
    double seconds = 0.0;
    long localCells = 0, localFaces = 0, localBounds = 0, localRegions = 0;
};

template <class Mesh, class Vec>
class BenchmarkKernels {
  public:
    using I = std::remove_cv_t<std::remove_reference_t<decltype(std::declval<Mesh &>().properties.lTCells)>>;
    using T = std::remove_cv_t<std::remove_reference_t<decltype(std::declval<Mesh &>().getFaceLambda(0))>>;

    // Arguments and contents of one GradientPhiGaussDolfyn call.
    struct GradientCall {
        I nGradient = 1;
        std::vector<T> phiCell, phiBoundary;
        std::vector<Vec> dPhidxCell, dPhidxoCell;
    };
    // Arguments and contents of one FluxMassDolfynFaceLoop call.
    struct MassCall {
        std::vector<Vec> dudx, dvdx, dwdx, dpdx;
        std::vector<T> denCell, denBoundary, uCell, vCell, wCell, massFlux, p, ar, su, rface;
        std::vector<T> teCell, teBoundary, edCell, edBoundary, viseffCell, viseffBoundary, tCell, tBoundary;
        T small = T(1e-18);
        I icinl = 0, icout = 0, icsym = 0, icwal = 0;
        bool solveTurbEnergy = false, solveTurbDiss = false, solveVisc = true, solveEnthalpy = false;
    };

    BenchmarkKernels(std::string benchmarkName, std::shared_ptr<Mesh> meshPtr, I repetitions,
                     unsigned seed = 20261203u)
        : benchmarkName(std::move(benchmarkName)), repetitions(repetitions), meshPtr(std::move(meshPtr)),
          eng_(seed) {}

    // BenchmarkConfigKernels: the name and repetitions of a "BenchmarkKernels"
    // entry of a CUP-CFD JSON configuration (cupcfd_gpu/config.hpp).
    BenchmarkKernels(const KernelBenchmarkConfig &cfg, std::shared_ptr<Mesh> meshPtr, unsigned seed = 20261203u)
        : BenchmarkKernels(cfg.benchmarkName, std::move(meshPtr), (I) cfg.repetitions, seed) {}

    void setupBenchmark() {}

    ecode_t runBenchmark() {
        for (I i = 0; i < repetitions; i++) {
            ecode_t (BenchmarkKernels::*steps[])() = {
                &BenchmarkKernels::GradientPhiGaussDolfynBenchmark, &BenchmarkKernels::FluxMassDolfynFaceLoopBenchmark,
                &BenchmarkKernels::FluxMassDolfynBoundaryLoop1Benchmark, &BenchmarkKernels::FluxMassDolfynBoundaryLoop2Benchmark,
                &BenchmarkKernels::FluxMassDolfynBoundaryLoop3Benchmark, &BenchmarkKernels::FluxMassDolfynBoundaryLoop4Benchmark,
                &BenchmarkKernels::FluxMassDolfynBoundaryLoop5Benchmark, &BenchmarkKernels::FluxMassDolfynRegionLoopBenchmark,
                &BenchmarkKernels::FluxUVWDolfynFaceLoop1Benchmark, &BenchmarkKernels::FluxUVWDolfynRegionLoop1Benchmark,
                &BenchmarkKernels::FluxUVWDolfynBndsLoop1Benchmark};
            for (auto s : steps) {
                ecode_t rc = (this->*s)();
                if ((int) rc != CUPCFD_E_SUCCESS) return rc;
            }
        }
        return (ecode_t) CUPCFD_E_SUCCESS;
    }

    ecode_t GradientPhiGaussDolfynBenchmark() {
        Mesh &mesh = *meshPtr;
        const I nCells = mesh.properties.lTCells, nBnds = mesh.properties.lBoundaries;
        GradientCall c;
        c.nGradient = 1;
        c.phiCell = uniform(nCells);
        c.phiBoundary = uniform(nBnds);
        c.dPhidxCell.resize((size_t) nCells);
        c.dPhidxoCell.resize((size_t) nCells);
        if (keep_) lastGradientIn_ = c;
        ecode_t rc = timed("GradientPhiGaussDolfynBenchmark", [&] {
            return cupcfd::fvm::gpu::GradientPhiGaussDolfyn(mesh, c.nGradient, c.phiCell.data(), nCells,
                                                            c.phiBoundary.data(), nBnds, c.dPhidxCell.data(), nCells,
                                                            c.dPhidxoCell.data(), nCells);
        });
        if (keep_) lastGradientOut_ = std::move(c);
        return rc;
    }

    ecode_t FluxMassDolfynFaceLoopBenchmark() {
        Mesh &mesh = *meshPtr;
        const I nCells = mesh.properties.lTCells, nBnds = mesh.properties.lBoundaries,
                nFaces = mesh.properties.lFaces;
        MassCall c;
        c.dudx = uniform_vec(nCells);
        c.dvdx = uniform_vec(nCells);
        c.dwdx = uniform_vec(nCells);
        c.dpdx = uniform_vec(nCells);
        c.denCell = uniform(nCells);
        c.denBoundary = uniform(nBnds);
        c.uCell = uniform(nCells);
        c.vCell = uniform(nCells);
        c.wCell = uniform(nCells);
        c.massFlux = uniform(nFaces);
        c.p = uniform(nCells);
        c.ar = uniform(nCells);
        c.su = uniform(nCells);
        c.rface.assign(2 * (size_t) nFaces, T(0));
        c.teCell = uniform(nCells);
        c.teBoundary = uniform(nBnds);
        c.edCell = uniform(nCells);
        c.edBoundary = uniform(nBnds);
        c.viseffCell = uniform(nCells);
        c.viseffBoundary = uniform(nBnds);
        c.tCell = uniform(nCells);
        c.tBoundary = uniform(nBnds);
        if (keep_) lastMassIn_ = c;
        ecode_t rc = timed("FluxMassDolfynFaceLoopBenchmark", [&] {
            return cupcfd::fvm::gpu::FluxMassDolfynFaceLoop(
                mesh, c.dudx.data(), nCells, c.dvdx.data(), nCells, c.dwdx.data(), nCells, c.dpdx.data(), nCells,
                c.denCell.data(), nCells, c.denBoundary.data(), nBnds, c.uCell.data(), nCells, c.vCell.data(), nCells,
                c.wCell.data(), nCells, c.massFlux.data(), nFaces, c.p.data(), nCells, c.ar.data(), nCells,
                c.su.data(), nCells, c.rface.data(), 2 * nFaces, c.small, &c.icinl, &c.icout, &c.icsym, &c.icwal,
                c.solveTurbEnergy, c.solveTurbDiss, c.solveVisc, c.solveEnthalpy, c.teCell.data(), nCells,
                c.teBoundary.data(), nBnds, c.edCell.data(), nCells, c.edBoundary.data(), nBnds,
                c.viseffCell.data(), nCells, c.viseffBoundary.data(), nBnds, c.tCell.data(), nCells,
                c.tBoundary.data(), nBnds);
        });
        if (keep_) lastMassOut_ = std::move(c);
        return rc;
    }

    ecode_t FluxMassDolfynBoundaryLoop1Benchmark() {
        Mesh &mesh = *meshPtr;
        const I nFaces = mesh.properties.lFaces;
        std::vector<T> massFlux = uniform(nFaces);
        T flowin = T(0);
        return timed("FluxMassDolfynBoundaryLoop1Benchmark", [&] {
            return cupcfd::fvm::gpu::FluxMassDolfynBoundaryLoop1(mesh, massFlux.data(), nFaces, &flowin);
        });
    }

    ecode_t FluxMassDolfynBoundaryLoop2Benchmark() {
        Mesh &mesh = *meshPtr;
        const I nFaces = mesh.properties.lFaces, nRegions = mesh.properties.lRegions;
        std::vector<T> massFlux = uniform(nFaces), flowRegion = uniform(nRegions);
        T flowout = T(0);
        return timed("FluxMassDolfynBoundaryLoop2Benchmark", [&] {
            return cupcfd::fvm::gpu::FluxMassDolfynBoundaryLoop2(mesh, massFlux.data(), nFaces, flowRegion.data(),
                                                                 nRegions, &flowout);
        });
    }

    ecode_t FluxMassDolfynBoundaryLoop3Benchmark() {
        Mesh &mesh = *meshPtr;
        T flowin = T(1.1), ratearea = T(0);
        return timed("FluxMassDolfynBoundaryLoop3Benchmark", [&] {
            return cupcfd::fvm::gpu::FluxMassDolfynBoundaryLoop3(mesh, flowin, &ratearea);
        });
    }

    ecode_t FluxMassDolfynBoundaryLoop4Benchmark() {
        Mesh &mesh = *meshPtr;
        const I nFaces = mesh.properties.lFaces, nBnds = mesh.properties.lBoundaries;
        std::vector<T> massFlux = uniform(nFaces), uB = uniform(nBnds), vB = uniform(nBnds), wB = uniform(nBnds),
                       denB = uniform(nBnds);
        T ratearea = T(1.0), flowout = T(0);
        return timed("FluxMassDolfynBoundaryLoop4Benchmark", [&] {
            return cupcfd::fvm::gpu::FluxMassDolfynBoundaryLoop4(mesh, massFlux.data(), nFaces, uB.data(), nBnds,
                                                                 vB.data(), nBnds, wB.data(), nBnds, denB.data(), nBnds,
                                                                 ratearea, &flowout);
        });
    }

    ecode_t FluxMassDolfynBoundaryLoop5Benchmark() {
        Mesh &mesh = *meshPtr;
        const I nFaces = mesh.properties.lFaces, nBnds = mesh.properties.lBoundaries,
                nCells = mesh.properties.lTCells, nRegions = mesh.properties.lRegions;
        std::vector<T> massFlux = uniform(nFaces), su = uniform(nCells), uB = uniform(nBnds), vB = uniform(nBnds),
                       wB = uniform(nBnds), flowFact = uniform(nRegions);
        T fact = T(1.1), flowout2 = T(0);
        return timed("FluxMassDolfynBoundaryLoop5Benchmark", [&] {
            return cupcfd::fvm::gpu::FluxMassDolfynBoundaryLoop5(mesh, massFlux.data(), nFaces, su.data(), nCells,
                                                                 uB.data(), nBnds, vB.data(), nBnds, wB.data(), nBnds,
                                                                 fact, true, true, true, flowFact.data(), nRegions,
                                                                 &flowout2);
        });
    }

    ecode_t FluxMassDolfynRegionLoopBenchmark() {
        Mesh &mesh = *meshPtr;
        const I nRegions = mesh.properties.lRegions;
        std::vector<T> flowFact = uniform(nRegions), flowRegion = uniform(nRegions);
        T flowIn = T(0.0);
        return timed("FluxMassDolfynRegionLoopBenchmark", [&] {
            return cupcfd::fvm::gpu::FluxMassDolfynRegionLoop(mesh, flowFact.data(), nRegions, flowRegion.data(),
                                                              nRegions, flowIn);
        });
    }

    ecode_t FluxUVWDolfynFaceLoop1Benchmark() {
        Mesh &mesh = *meshPtr;
        const I nCells = mesh.properties.lTCells, nBnds = mesh.properties.lBoundaries,
                nFaces = mesh.properties.lFaces;
        const T gammaBlend = T(0.9), small = T(1e-18);
        std::vector<T> u = uniform(nCells), v = uniform(nCells), w = uniform(nCells), vis = uniform(nCells),
                       mf = uniform(nFaces), su = uniform(nCells), sv = uniform(nCells), sw = uniform(nCells),
                       au = uniform(nCells), av = uniform(nCells), aw = uniform(nCells);
        std::vector<Vec> dudx = uniform_vec(nCells), dvdx = uniform_vec(nCells), dwdx = uniform_vec(nCells);
        std::vector<T> uB = uniform(nBnds), vB = uniform(nBnds), wB = uniform(nBnds), visB = uniform(nBnds);
        std::vector<T> rFace(2 * (size_t) nFaces, T(0));
        return timed("FluxUVWDolfynFaceLoop1Benchmark", [&] {
            return cupcfd::fvm::gpu::FluxUVWDolfynFaceLoop1(
                mesh, gammaBlend, small, u.data(), nCells, v.data(), nCells, w.data(), nCells, uB.data(), nBnds,
                vB.data(), nBnds, wB.data(), nBnds, vis.data(), nCells, visB.data(), nBnds, mf.data(), nFaces,
                dudx.data(), nCells, dvdx.data(), nCells, dwdx.data(), nCells, rFace.data(), 2 * nFaces, su.data(),
                nCells, sv.data(), nCells, sw.data(), nCells, au.data(), nCells, av.data(), nCells, aw.data(), nCells);
        });
    }

    ecode_t FluxUVWDolfynRegionLoop1Benchmark() {
        Mesh &mesh = *meshPtr;
        return timed("FluxUVWDolfynRegionLoop1Benchmark",
                     [&] { return cupcfd::fvm::gpu::FluxUVWDolfynRegionLoop1(mesh); });
    }

    ecode_t FluxUVWDolfynBndsLoop1Benchmark() {
        Mesh &mesh = *meshPtr;
        return timed("FluxUVWDolfynBndsLoop1Benchmark", [&] { return cupcfd::fvm::gpu::FluxUVWDolfynBndsLoop1(mesh); });
    }

    // every timed call so far, in call order
    const std::vector<Timing> &timings() const { return timings_; }

    // keep the inputs and results of the latest GradientPhiGaussDolfyn and
    // FluxMassDolfynFaceLoop calls (off by default: they double the memory)
    void keepLastCalls(bool on) { keep_ = on; }
    const GradientCall &lastGradientInputs() const { return lastGradientIn_; }
    const GradientCall &lastGradientResults() const { return lastGradientOut_; }
    const MassCall &lastMassInputs() const { return lastMassIn_; }
    const MassCall &lastMassResults() const { return lastMassOut_; }

    std::string benchmarkName;
    I repetitions;
    std::shared_ptr<Mesh> meshPtr;

  private:
    std::default_random_engine eng_;
    std::vector<Timing> timings_;
    bool keep_ = false;
    GradientCall lastGradientIn_, lastGradientOut_;
    MassCall lastMassIn_, lastMassOut_;

    std::vector<T> uniform(I n) {
        std::uniform_real_distribution<double> unif(1e-6, 1e-2);
        std::vector<T> v((size_t) n);
        for (T &x : v) x = (T) unif(eng_);
        return v;
    }
    std::vector<Vec> uniform_vec(I n) {
        std::uniform_real_distribution<double> unif(1e-6, 1e-2);
        std::vector<Vec> v((size_t) n);
        for (Vec &x : v)
            for (int d = 0; d < 3; d++) x.cmp[d] = (T) unif(eng_);
        return v;
    }
    template <class F>
    ecode_t timed(const char *name, F &&call) {
        Mesh &mesh = *meshPtr;
        // the first call on a mesh uploads it: done before the clock starts,
        // as the reference builds its mesh outside its timers
        cupcfd_gpu_mesh *m = nullptr;
        int up = cupcfd::fvm::gpu::attach(mesh, &m);
        if (up != CUPCFD_E_SUCCESS) return (ecode_t) up;
        const auto t0 = std::chrono::steady_clock::now();
        ecode_t rc = call();
        const auto t1 = std::chrono::steady_clock::now();
        Timing t;
        t.name = name;
        t.seconds = std::chrono::duration<double>(t1 - t0).count();
        t.localCells = (long) mesh.properties.lTCells;
        t.localFaces = (long) mesh.properties.lFaces;
        t.localBounds = (long) mesh.properties.lBoundaries;
        t.localRegions = (long) mesh.properties.lRegions;
        timings_.push_back(t);
        return rc;
    }
};

}  // namespace gpu
}  // namespace benchmark
}  // namespace cupcfd
