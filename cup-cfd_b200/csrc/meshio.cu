// Mesh files: a raw-binary copy of a device mesh's source arrays, so a mesh
// built once (from a MeshSource-like generator, or uploaded from a host
// CupCfdSoAMesh) can be reloaded without its original source. The
// reference reads meshes through MeshHDF5Source (HDF5 datasets, not
// available in this build); this format holds the same per-face and
// per-cell quantities in the reference's numbering, and loading rebuilds
// the device layout with cupcfd_gpu_mesh_create.
//
// Layout (little-endian): a 64-byte header
//   char magic[8] = "CUPCFDM1"; int32 version = 1; int32 nCells, nFaces,
//   nBoundaries, nRegions; int32 flags (bit 0: xpac/xnac present, bit 1:
//   rlencos present, bit 2: boundary distances present);
//   int32 reserved[8] = 0
// then, in this order, faceCell1, faceCell2, faceBnd [nFaces] int32;
// faceLambda, faceArea [nFaces] and faceNorm, faceCenter [3 nFaces] float64;
// faceXpac, faceXnac [3 nFaces] float64 when flags bit 0 is set; cellCenter [3 nCells],
// cellVolume [nCells] float64; regionType [nRegions] int32, regionUVW
// [3 nRegions], regionDen, regionSplvl [nRegions] float64; bndRegion
// [nBoundaries] int32; faceRLencos [nFaces] float64 when flags bit 1 is set;
// boundaryDistance [nBoundaries] float64 when flags bit 2 is set; and last
// the FNV-1a 64-bit hash of everything before it.
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "internal.cuh"

using namespace cupcfd_gpu;

namespace {

constexpr char MAGIC[8] = {'C', 'U', 'P', 'C', 'F', 'D', 'M', '1'};
constexpr int VERSION = 2;  // 2: word-wise checksum

struct Header {
    char magic[8];
    int32_t version, nCells, nFaces, nBnd, nRegions, flags;
    int32_t reserved[8];
};
static_assert(sizeof(Header) == 64, "64-byte header");

// FNV-1a over the little-endian 64-bit words of the byte stream (the stream
// is every byte added, in order; a last partial word is padded with zero
// bytes): h = (h ^ word) * prime. A step per eight bytes instead of one per
// byte; value() is the hash of everything added.
struct Fnv {
    uint64_t h = 1469598103934665603ULL;
    unsigned char pend[8] = {0};
    size_t npend = 0;
    void word(uint64_t w) {
        h ^= w;
        h *= 1099511628211ULL;
    }
    void add(const void *p, size_t n) {
        const unsigned char *b = (const unsigned char *) p;
        while (n > 0 && npend > 0) {  // complete a pending word
            pend[npend++] = *b++;
            n--;
            if (npend == 8) {
                uint64_t w;
                std::memcpy(&w, pend, 8);
                word(w);
                npend = 0;
            }
        }
        for (; n >= 8; n -= 8, b += 8) {
            uint64_t w;
            std::memcpy(&w, b, 8);
            word(w);
        }
        for (; n > 0; n--) pend[npend++] = *b++;
    }
    uint64_t value() const {
        if (npend == 0) return h;
        unsigned char last[8] = {0};
        std::memcpy(last, pend, npend);
        uint64_t w;
        std::memcpy(&w, last, 8);
        return (h ^ w) * 1099511628211ULL;
    }
};

struct File {
    FILE *f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};

template <class T>
bool put(File &fl, Fnv &h, const std::vector<T> &v) {
    h.add(v.data(), v.size() * sizeof(T));
    return v.empty() || fwrite(v.data(), sizeof(T), v.size(), fl.f) == v.size();
}

template <class T>
bool get(File &fl, Fnv &h, std::vector<T> &v, size_t n) {
    v.resize(n);
    if (n && fread(v.data(), sizeof(T), n, fl.f) != n) return false;
    h.add(v.data(), n * sizeof(T));
    return true;
}

template <class T>
int download(std::vector<T> &out, const T *dev, size_t n, cudaStream_t st) {
    out.resize(n);
    if (n) CG_CHECK_CUDA(cudaMemcpyAsync(out.data(), dev, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    return CUPCFD_E_SUCCESS;
}

}  // namespace

namespace {
int mesh_save(const cupcfd_gpu_mesh *m, const char *path) {
    CG_RETURN_IF(!m || !path, CUPCFD_E_NULL_PTR, "mesh_save: null argument");
    CG_TRY(make_device_current(m->device));
    const int nC = m->nC, nF = m->nF, nB = m->nB, nR = m->nR;
    std::vector<int32_t> c1(nF), c2(nF), bnd(nF);
    std::vector<double> lam(nF), area(nF), S(3 * (size_t) nF), X(3 * (size_t) nF), cc(3 * (size_t) nC), vol(nC);
    CG_TRY(cupcfd_gpu_mesh_get_geometry(m, c1.data(), c2.data(), bnd.data(), lam.data(), area.data(), S.data(),
                                        X.data(), cc.data(), vol.data()));
    cudaStream_t st = m->stream;
    std::vector<double> xp, xn;
    int flags = 0;
    if (!m->xpacZero) {  // internal double4 records -> reference order, xyz
        flags |= 1;
        std::vector<double4> a, b;
        std::vector<int> n2o;
        CG_TRY(download(a, m->fxp64, (size_t) nF, st));
        CG_TRY(download(b, m->fxn64, (size_t) nF, st));
        CG_TRY(download(n2o, (const int *) m->faceN2O, (size_t) nF, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        xp.resize(3 * (size_t) nF);
        xn.resize(3 * (size_t) nF);
        for (int f = 0; f < nF; f++) {
            size_t o = 3 * (size_t) n2o[f];
            xp[o] = a[f].x; xp[o + 1] = a[f].y; xp[o + 2] = a[f].z;
            xn[o] = b[f].x; xn[o + 1] = b[f].y; xn[o + 2] = b[f].z;
        }
    }
    std::vector<double> rl, bd;  // momentum-loop geometry, when set
    if (m->rlencos) {
        flags |= 2;
        std::vector<double> a;
        std::vector<int> n2o;
        CG_TRY(download(a, (const double *) m->rlencos, (size_t) nF, st));
        CG_TRY(download(n2o, (const int *) m->faceN2O, (size_t) nF, st));
        CG_CHECK_CUDA(cudaStreamSynchronize(st));
        rl.resize(nF);
        for (int f = 0; f < nF; f++) rl[n2o[f]] = a[f];
    }
    if (m->bndDist) {
        flags |= 4;
        CG_TRY(download(bd, (const double *) m->bndDist, (size_t) nB, st));
    }
    std::vector<int32_t> rtype(m->hRegionType.begin(), m->hRegionType.end()), breg;
    std::vector<double> ruvw, rden, rsp;
    CG_TRY(download(ruvw, (const double *) m->regionUVW, 3 * (size_t) nR, st));
    CG_TRY(download(rden, (const double *) m->regionDen, (size_t) nR, st));
    CG_TRY(download(rsp, (const double *) m->regionSplvl, (size_t) nR, st));
    CG_TRY(download(breg, (const int32_t *) m->bndRegion, (size_t) nB, st));
    CG_CHECK_CUDA(cudaStreamSynchronize(st));

    File fl;
    fl.f = fopen(path, "wb");
    CG_RETURN_IF(!fl.f, CUPCFD_E_FILE_MISSING, std::string("mesh_save: cannot open ") + path + " for writing");
    Header hd;
    std::memset(&hd, 0, sizeof(hd));
    std::memcpy(hd.magic, MAGIC, 8);
    hd.version = VERSION;
    hd.nCells = nC; hd.nFaces = nF; hd.nBnd = nB; hd.nRegions = nR; hd.flags = flags;
    Fnv h;
    h.add(&hd, sizeof(hd));
    bool ok = fwrite(&hd, sizeof(hd), 1, fl.f) == 1;
    ok = ok && put(fl, h, c1) && put(fl, h, c2) && put(fl, h, bnd) && put(fl, h, lam) && put(fl, h, area) &&
         put(fl, h, S) && put(fl, h, X);
    if (flags & 1) ok = ok && put(fl, h, xp) && put(fl, h, xn);
    ok = ok && put(fl, h, cc) && put(fl, h, vol) && put(fl, h, rtype) && put(fl, h, ruvw) && put(fl, h, rden) &&
         put(fl, h, rsp) && put(fl, h, breg);
    if (flags & 2) ok = ok && put(fl, h, rl);
    if (flags & 4) ok = ok && put(fl, h, bd);
    const uint64_t sum = h.value();
    ok = ok && fwrite(&sum, sizeof(sum), 1, fl.f) == 1;
    CG_RETURN_IF(!ok, CUPCFD_E_ERROR, std::string("mesh_save: write to ") + path + " failed");
    CG_RETURN_IF(fclose(fl.f) != 0, CUPCFD_E_ERROR, std::string("mesh_save: closing ") + path + " failed");
    fl.f = nullptr;
    return CUPCFD_E_SUCCESS;
}

int mesh_load(const char *path, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) {
    CG_RETURN_IF(!path || !out, CUPCFD_E_NULL_PTR, "mesh_load: null argument");
    *out = nullptr;
    File fl;
    fl.f = fopen(path, "rb");
    CG_RETURN_IF(!fl.f, CUPCFD_E_FILE_MISSING, std::string("mesh_load: cannot open ") + path);
    Header hd;
    CG_RETURN_IF(fread(&hd, sizeof(hd), 1, fl.f) != 1 || std::memcmp(hd.magic, MAGIC, 8) != 0,
                 CUPCFD_E_INVALID_FILE_FORMAT, std::string("mesh_load: ") + path + " is not a mesh file");
    CG_RETURN_IF(hd.version != VERSION, CUPCFD_E_INVALID_FILE_FORMAT, "mesh_load: unknown format version");
    CG_RETURN_IF(hd.nCells < 1 || hd.nFaces < 1 || hd.nBnd < 0 || hd.nRegions < 1 || (hd.flags & ~7) != 0,
                 CUPCFD_E_INVALID_FILE_FORMAT, "mesh_load: header out of range");
    const size_t nC = hd.nCells, nF = hd.nFaces, nB = hd.nBnd, nR = hd.nRegions;
    // the size the header implies, checked before anything is allocated
    size_t want = sizeof(Header) + nF * (3 * 4 + 2 * 8 + 6 * 8) + ((hd.flags & 1) ? nF * 6 * 8 : 0) + nC * 4 * 8 +
                  nR * (4 + 5 * 8) + nB * 4 + ((hd.flags & 2) ? nF * 8 : 0) + ((hd.flags & 4) ? nB * 8 : 0) +
                  sizeof(uint64_t);
    CG_RETURN_IF(fseek(fl.f, 0, SEEK_END) != 0, CUPCFD_E_ERROR, "mesh_load: cannot seek");
    long have = ftell(fl.f);
    CG_RETURN_IF(have < 0 || (size_t) have != want, CUPCFD_E_INVALID_FILE_FORMAT,
                 std::string("mesh_load: ") + path + " has the wrong size for its header");
    CG_RETURN_IF(fseek(fl.f, (long) sizeof(Header), SEEK_SET) != 0, CUPCFD_E_ERROR, "mesh_load: cannot seek");
    Fnv h;
    h.add(&hd, sizeof(hd));
    std::vector<int32_t> c1, c2, bnd, rtype, breg;
    std::vector<double> lam, area, S, X, xp, xn, cc, vol, ruvw, rden, rsp, rl, bd;
    bool ok = get(fl, h, c1, nF) && get(fl, h, c2, nF) && get(fl, h, bnd, nF) && get(fl, h, lam, nF) &&
              get(fl, h, area, nF) && get(fl, h, S, 3 * nF) && get(fl, h, X, 3 * nF);
    if (hd.flags & 1) ok = ok && get(fl, h, xp, 3 * nF) && get(fl, h, xn, 3 * nF);
    ok = ok && get(fl, h, cc, 3 * nC) && get(fl, h, vol, nC) && get(fl, h, rtype, nR) && get(fl, h, ruvw, 3 * nR) &&
         get(fl, h, rden, nR) && get(fl, h, rsp, nR) && get(fl, h, breg, nB);
    if (hd.flags & 2) ok = ok && get(fl, h, rl, nF);
    if (hd.flags & 4) ok = ok && get(fl, h, bd, nB);
    uint64_t stored = 0;
    ok = ok && fread(&stored, sizeof(stored), 1, fl.f) == 1;
    CG_RETURN_IF(!ok, CUPCFD_E_INVALID_FILE_FORMAT, std::string("mesh_load: ") + path + " is truncated");
    CG_RETURN_IF(stored != h.value(), CUPCFD_E_INVALID_FILE_FORMAT, std::string("mesh_load: checksum mismatch in ") + path);

    cupcfd_mesh_view v;
    std::memset(&v, 0, sizeof(v));
    v.nCells = (int32_t) nC; v.nFaces = (int32_t) nF; v.nBoundaries = (int32_t) nB; v.real_size = sizeof(double);
    v.faceCell1 = c1.data(); v.faceCell2 = c2.data(); v.faceBnd = bnd.data();
    v.faceLambda = lam.data(); v.faceArea = area.data(); v.cellVolume = vol.data();
    v.faceNorm = {S.data(), (int32_t) (3 * sizeof(double)), 0};
    v.faceCenter = {X.data(), (int32_t) (3 * sizeof(double)), 0};
    v.faceXpac = {xp.empty() ? nullptr : xp.data(), (int32_t) (3 * sizeof(double)), 0};
    v.faceXnac = {xn.empty() ? nullptr : xn.data(), (int32_t) (3 * sizeof(double)), 0};
    v.cellCenter = {cc.data(), (int32_t) (3 * sizeof(double)), 0};
    cupcfd_gpu_mesh *m = nullptr;
    CG_TRY(cupcfd_gpu_mesh_create(&v, opt, &m));
    int rc = cupcfd_gpu_mesh_set_regions(m, (int32_t) nR, rtype.data(), ruvw.data(), rden.data(), breg.data(),
                                         (int32_t) nB);
    if (rc == CUPCFD_E_SUCCESS) rc = cupcfd_gpu_mesh_set_region_split(m, (int32_t) nR, rsp.data());
    if (rc == CUPCFD_E_SUCCESS && !rl.empty()) rc = cupcfd_gpu_mesh_set_face_rlencos(m, rl.data(), (int32_t) nF);
    if (rc == CUPCFD_E_SUCCESS && (hd.flags & 4)) rc = cupcfd_gpu_mesh_set_boundary_distance(m, bd.data(), (int32_t) nB);
    if (rc != CUPCFD_E_SUCCESS) {
        std::string msg = cupcfd_gpu_last_error();
        cupcfd_gpu_mesh_destroy(m);
        set_error("mesh_load: " + msg);
        return rc;
    }
    *out = m;
    return CUPCFD_E_SUCCESS;
}
}  // namespace

extern "C" int cupcfd_gpu_mesh_save(const cupcfd_gpu_mesh *m, const char *path) {
    clear_error();
    try {
        return mesh_save(m, path);
    } catch (const std::exception &e) {
        set_error(std::string("mesh_save: ") + e.what());
        return CUPCFD_E_ERROR;
    }
}

extern "C" int cupcfd_gpu_mesh_load(const char *path, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) {
    clear_error();
    try {
        return mesh_load(path, opt, out);
    } catch (const std::exception &e) {
        set_error(std::string("mesh_load: ") + e.what());
        return CUPCFD_E_ERROR;
    }
}
