// On-GPU mesh sources in the reference's label order, FP64.
//
// Structured: MeshStructGenSource (src/geometry/mesh/implementation/source/
// MeshStructGenSource.cpp) -- labels, connectivity, lambda, face normals
// (clockwise test from cell1's centre), Heron-fan areas and centroids, cell
// centres. Every floating-point operation is an explicit round-to-nearest
// intrinsic in the reference's operand order, so no FMA contraction changes
// the rounding: the arrays equal those of the reference generator bit for
// bit, except cell volumes (box volume here; the reference sums five Heron
// tetrahedra, Hexahedron.ipp:135-139, which agrees to 2e-14 relative).
//
// Jittered: the irregular-mesh geometry documented in cupcfd_gpu.h.
#include <cub/cub.cuh>

#include <vector>

#include "internal.cuh"

namespace cupcfd_gpu {
int mesh_new(const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out);
}

namespace {
using namespace cupcfd_gpu;

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dv(double a, double b) { return __ddiv_rn(a, b); }

struct V3 {
    double x, y, z;
};
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return {ds(a.x, b.x), ds(a.y, b.y), ds(a.z, b.z)}; }
// dotP = 0; dotP += a_i * b_i   (EuclideanVector.cpp:83-90)
__device__ __forceinline__ double dot(V3 a, V3 b) {
    double d = 0.0;
    d = da(d, dm(a.x, b.x));
    d = da(d, dm(a.y, b.y));
    d = da(d, dm(a.z, b.z));
    return d;
}
// EuclideanVector3D.ipp:55-63
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {ds(dm(a.y, b.z), dm(a.z, b.y)), ds(dm(a.z, b.x), dm(a.x, b.z)), ds(dm(a.x, b.y), dm(a.y, b.x))};
}
__device__ __forceinline__ double len(V3 v) { return __dsqrt_rn(dot(v, v)); }
// Triangle.ipp:83-99
__device__ __forceinline__ double heron(V3 a, V3 b, V3 c) {
    double ab = len(sub(b, a)), ac = len(sub(c, a)), bc = len(sub(c, b));
    double s = dv(da(da(ab, ac), bc), 2.0);
    return __dsqrt_rn(dm(dm(dm(s, ds(s, ab)), ds(s, bc)), ds(s, ac)));
}

struct Grid {
    int nx, ny, nz;
    double sx, sy, sz, hx, hy, hz;
    int nYZ, nXZ, nBYZ, nBXZ;
};

__device__ __forceinline__ int gcell(const Grid &g, int x, int y, int z) { return x + y * g.nx + z * g.nx * g.ny; }
__device__ __forceinline__ int gvert(const Grid &g, int x, int y, int z) {
    return x + y * (g.nx + 1) + z * (g.nx + 1) * (g.ny + 1);
}

// face label -> orientation and integer coordinates (MeshStructGenSource.cpp:449-500)
__device__ void face_coords(const Grid &g, int f, int &k, int &x, int &y, int &z) {
    if (f < g.nYZ) {
        k = 0; x = f % (g.nx + 1); y = (f / (g.nx + 1)) % g.ny; z = f / ((g.nx + 1) * g.ny);
    } else if (f < g.nYZ + g.nXZ) {
        int l = f - g.nYZ;
        k = 1; x = l % g.nx; y = (l / g.nx) % (g.ny + 1); z = l / (g.nx * (g.ny + 1));
    } else {
        int l = f - g.nYZ - g.nXZ;
        k = 2; x = l % g.nx; y = (l / g.nx) % g.ny; z = l / (g.nx * g.ny);
    }
}

// getFaceCell1Labels / getFaceCell2Labels / getFaceBoundaryLabels (:516-822)
__device__ void face_conn(const Grid &g, int f, int &c1, int &c2, int &bl) {
    int k, x, y, z;
    face_coords(g, f, k, x, y, z);
    if (k == 0) {
        bool lo = x == 0, hi = x == g.nx;
        c1 = gcell(g, lo ? x : x - 1, y, z);
        c2 = (lo || hi) ? -1 : gcell(g, x, y, z);
        bl = lo ? (y * 2 + z * 2 * g.ny) : hi ? (1 + y * 2 + z * 2 * g.ny) : -1;
    } else if (k == 1) {
        bool lo = y == 0, hi = y == g.ny;
        c1 = gcell(g, x, lo ? y : y - 1, z);
        c2 = (lo || hi) ? -1 : gcell(g, x, y, z);
        bl = lo ? (g.nBYZ + x + z * g.nx * 2) : hi ? (g.nBYZ + x + g.nx + z * g.nx * 2) : -1;
    } else {
        bool lo = z == 0, hi = z == g.nz;
        c1 = gcell(g, x, y, lo ? z : z - 1);
        c2 = (lo || hi) ? -1 : gcell(g, x, y, z);
        bl = lo ? (g.nBYZ + g.nBXZ + x + y * g.nx) : hi ? (g.nBYZ + g.nBXZ + x + y * g.nx + g.nx * g.ny) : -1;
    }
}

// getFaceVerticesLabelsCSR (:980-1084)
__device__ void face_verts(const Grid &g, int f, int *v) {
    int k, x, y, z;
    face_coords(g, f, k, x, y, z);
    if (k == 0) {
        v[0] = gvert(g, x, y, z); v[1] = gvert(g, x, y + 1, z); v[2] = gvert(g, x, y + 1, z + 1); v[3] = gvert(g, x, y, z + 1);
    } else if (k == 1) {
        v[0] = gvert(g, x, y, z); v[1] = gvert(g, x + 1, y, z); v[2] = gvert(g, x + 1, y, z + 1); v[3] = gvert(g, x, y, z + 1);
    } else {
        v[0] = gvert(g, x, y, z); v[1] = gvert(g, x + 1, y, z); v[2] = gvert(g, x + 1, y + 1, z); v[3] = gvert(g, x, y + 1, z);
    }
}

// getVertexCoords (:1086-1112)
__device__ V3 vert_coords(const Grid &g, int v) {
    int x = v % (g.nx + 1), y = (v / (g.nx + 1)) % (g.ny + 1), z = v / ((g.nx + 1) * (g.ny + 1));
    return {da(g.sx, dm(g.hx, (double) x)), da(g.sy, dm(g.hy, (double) y)), da(g.sz, dm(g.hz, (double) z))};
}

// getCellCenter (:323-354) and the box bounds used for the volume
__device__ V3 cell_center(const Grid &g, int c, V3 *lo, V3 *hi) {
    int x = c % g.nx, y = (c / g.nx) % g.ny, z = c / (g.nx * g.ny);
    V3 l = {da(g.sx, dm((double) x, g.hx)), da(g.sy, dm((double) y, g.hy)), da(g.sz, dm((double) z, g.hz))};
    V3 h = {da(g.sx, dm((double) (x + 1), g.hx)), da(g.sy, dm((double) (y + 1), g.hy)), da(g.sz, dm((double) (z + 1), g.hz))};
    if (lo) *lo = l;
    if (hi) *hi = h;
    return {da(l.x, dv(ds(h.x, l.x), 2.0)), da(l.y, dv(ds(h.y, l.y), 2.0)), da(l.z, dv(ds(h.z, l.z), 2.0))};
}

__global__ void k_structgen_cells(Grid g, int nC, double *__restrict__ cc, double *__restrict__ vol) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    V3 lo, hi;
    V3 p = cell_center(g, c, &lo, &hi);
    cc[3 * c] = p.x; cc[3 * c + 1] = p.y; cc[3 * c + 2] = p.z;
    vol[c] = dm(dm(ds(hi.x, lo.x), ds(hi.y, lo.y)), ds(hi.z, lo.z));
}

__global__ void k_structgen_faces(Grid g, int nF, int *__restrict__ c1o, int *__restrict__ c2o, int *__restrict__ bo,
                                  double *__restrict__ lam, double *__restrict__ area, double *__restrict__ S,
                                  double *__restrict__ xf) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int c1, c2, bl, vl[4];
    face_conn(g, f, c1, c2, bl);
    c1o[f] = c1; c2o[f] = c2; bo[f] = bl;
    lam[f] = bl >= 0 ? -1.0 : 0.5;  // getFaceLambda (:824-850)
    face_verts(g, f, vl);
    V3 P[4];
    for (int k = 0; k < 4; k++) P[k] = vert_coords(g, vl[k]);
    // Polygon3D::computeArea / computeCentroid (Polygon3D.cpp:31-55)
    double a1 = heron(P[0], P[1], P[2]);
    double a2 = heron(P[0], P[2], P[3]);
    double A = da(da(0.0, a1), a2);
    double t1x = dv(da(da(P[0].x, P[1].x), P[2].x), 3.0), t2x = dv(da(da(P[0].x, P[2].x), P[3].x), 3.0);
    double t1y = dv(da(da(P[0].y, P[1].y), P[2].y), 3.0), t2y = dv(da(da(P[0].y, P[2].y), P[3].y), 3.0);
    double t1z = dv(da(da(P[0].z, P[1].z), P[2].z), 3.0), t2z = dv(da(da(P[0].z, P[2].z), P[3].z), 3.0);
    xf[3 * f] = dv(da(da(0.0, dm(t1x, a1)), dm(t2x, a2)), A);
    xf[3 * f + 1] = dv(da(da(0.0, dm(t1y, a1)), dm(t2y, a2)), A);
    xf[3 * f + 2] = dv(da(da(0.0, dm(t1z, a1)), dm(t2z, a2)), A);
    area[f] = A;
    // getFaceNormal (:887-946), isVertexOrderClockwise (Polygon3D.cpp:93-119)
    V3 obs = cell_center(g, c1, nullptr, nullptr);
    V3 nn = cross(sub(P[1], P[0]), sub(P[2], P[0]));
    V3 n = dot(nn, sub(obs, P[0])) < 0.0 ? nn : cross(sub(P[1], P[2]), sub(P[0], P[2]));
    S[3 * f] = n.x; S[3 * f + 1] = n.y; S[3 * f + 2] = n.z;
}

// ---------------------------------------------------------------------------
// jittered mesh
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

__device__ __forceinline__ double hash_unit(unsigned long long seed, unsigned long long key) {
    unsigned long long r = splitmix64(seed ^ splitmix64(key));
    return ds(dm(dm((double) (r >> 11), 1.0 / 9007199254740992.0), 2.0), 1.0);
}

__global__ void k_jit_verts(Grid g, int nV, double jitter, unsigned long long seed, double *__restrict__ vc) {
    int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nV) return;
    int x = v % (g.nx + 1), y = (v / (g.nx + 1)) % (g.ny + 1), z = v / ((g.nx + 1) * (g.ny + 1));
    V3 p = vert_coords(g, v);
    double q[3] = {p.x, p.y, p.z}, h[3] = {g.hx, g.hy, g.hz};
    bool interior = x > 0 && x < g.nx && y > 0 && y < g.ny && z > 0 && z < g.nz;
    if (interior)
        for (int d = 0; d < 3; d++) q[d] = da(q[d], dm(dm(jitter, h[d]), hash_unit(seed, 3ULL * (unsigned long long) v + d)));
    vc[3 * v] = q[0]; vc[3 * v + 1] = q[1]; vc[3 * v + 2] = q[2];
}

__global__ void k_jit_centres(Grid g, int nC, const double *__restrict__ vc, double *__restrict__ cc) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int x = c % g.nx, y = (c / g.nx) % g.ny, z = c / (g.nx * g.ny);
    double s[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 8; k++) {
        int v = gvert(g, x + (k & 1), y + ((k >> 1) & 1), z + ((k >> 2) & 1));
        for (int d = 0; d < 3; d++) s[d] = da(s[d], vc[3 * v + d]);
    }
    for (int d = 0; d < 3; d++) cc[3 * c + d] = dv(s[d], 8.0);
}

__global__ void k_jit_faces(Grid g, int nF, const double *__restrict__ vc, const double *__restrict__ cc,
                            int *__restrict__ f1, int *__restrict__ f2, double *__restrict__ lam, double *__restrict__ area,
                            double *__restrict__ S, double *__restrict__ xf, double *__restrict__ dvol) {
    int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nF) return;
    int c1, c2, bl, vl[4];
    face_conn(g, f, c1, c2, bl);
    f1[f] = c1; f2[f] = c2;
    face_verts(g, f, vl);
    V3 p[4];
    for (int k = 0; k < 4; k++) p[k] = {vc[3 * vl[k]], vc[3 * vl[k] + 1], vc[3 * vl[k] + 2]};
    V3 s = cross(sub(p[2], p[0]), sub(p[3], p[1]));
    s = {dm(0.5, s.x), dm(0.5, s.y), dm(0.5, s.z)};
    V3 x = {dv(da(da(da(p[0].x, p[1].x), p[2].x), p[3].x), 4.0), dv(da(da(da(p[0].y, p[1].y), p[2].y), p[3].y), 4.0),
            dv(da(da(da(p[0].z, p[1].z), p[2].z), p[3].z), 4.0)};
    V3 cP = {cc[3 * c1], cc[3 * c1 + 1], cc[3 * c1 + 2]};
    if (dot(s, sub(x, cP)) < 0.0) s = {-s.x, -s.y, -s.z};
    S[3 * f] = s.x; S[3 * f + 1] = s.y; S[3 * f + 2] = s.z;
    xf[3 * f] = x.x; xf[3 * f + 1] = x.y; xf[3 * f + 2] = x.z;
    area[f] = len(s);
    dvol[f] = dv(dot(x, s), 3.0);
    if (c2 >= 0) {
        V3 cN = {cc[3 * c2], cc[3 * c2 + 1], cc[3 * c2 + 2]};
        lam[f] = dv(dot(sub(x, cP), s), dot(sub(cN, cP), s));
    } else {
        lam[f] = -1.0;
    }
}

// a cell's six faces in ascending label: YZ low/high, XZ low/high, XY low/high
__global__ void k_jit_volumes(Grid g, int nC, const int *__restrict__ f1, const double *__restrict__ dvol,
                              double *__restrict__ vol) {
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nC) return;
    int x = c % g.nx, y = (c / g.nx) % g.ny, z = c / (g.nx * g.ny);
    int fl[6] = {x + y * (g.nx + 1) + z * (g.nx + 1) * g.ny, (x + 1) + y * (g.nx + 1) + z * (g.nx + 1) * g.ny,
                 g.nYZ + x + y * g.nx + z * g.nx * (g.ny + 1), g.nYZ + x + (y + 1) * g.nx + z * g.nx * (g.ny + 1),
                 g.nYZ + g.nXZ + x + y * g.nx + z * g.nx * g.ny, g.nYZ + g.nXZ + x + y * g.nx + (z + 1) * g.nx * g.ny};
    double v = 0.0;
    for (int k = 0; k < 6; k++) v = (f1[fl[k]] == c) ? da(v, dvol[fl[k]]) : ds(v, dvol[fl[k]]);
    vol[c] = v;
}

__global__ void k_jit_permute(int nC, int nF, const int *__restrict__ cp, const int *__restrict__ fp,
                              const int *__restrict__ f1, const int *__restrict__ f2, const double *__restrict__ lam,
                              const double *__restrict__ area, const double *__restrict__ S, const double *__restrict__ xf,
                              const double *__restrict__ cc, const double *__restrict__ vol, int *__restrict__ o1,
                              int *__restrict__ o2, int *__restrict__ isB, double *__restrict__ olam,
                              double *__restrict__ oarea, double *__restrict__ oS, double *__restrict__ oxf,
                              double *__restrict__ occ, double *__restrict__ ovol) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nF) {
        int n = fp[i];
        o1[n] = cp[f1[i]];
        o2[n] = f2[i] >= 0 ? cp[f2[i]] : -1;
        isB[n] = f2[i] < 0 ? 1 : 0;
        olam[n] = lam[i];
        oarea[n] = area[i];
        for (int d = 0; d < 3; d++) { oS[3 * n + d] = S[3 * i + d]; oxf[3 * n + d] = xf[3 * i + d]; }
    }
    if (i < nC) {
        int n = cp[i];
        for (int d = 0; d < 3; d++) occ[3 * n + d] = cc[3 * i + d];
        ovol[n] = vol[i];
    }
}

__global__ void k_bnd_ids(int nF, const int *__restrict__ isB, const int *__restrict__ scan, int *__restrict__ bnd) {
    int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n < nF) bnd[n] = isB[n] ? scan[n] : -1;
}

void host_shuffle(std::vector<int> &p, unsigned long long seed) {
    int n = (int) p.size();
    for (int i = 0; i < n; i++) p[i] = i;
    unsigned long long s = seed;
    for (int i = n - 1; i > 0; i--) {
        s = splitmix64(s);
        int j = (int) (s % (unsigned long long) (i + 1));
        std::swap(p[i], p[j]);
    }
}

struct Pool {
    std::vector<void *> p;
    ~Pool() { for (void *q : p) cudaFree(q); }
    template <class T>
    T *get(size_t n) {
        void *q = nullptr;
        if (cudaMalloc(&q, (n ? n : 1) * sizeof(T)) != cudaSuccess) return nullptr;
        p.push_back(q);
        return (T *) q;
    }
};

Grid make_grid(int nx, int ny, int nz, const double b[6]) {
    Grid g;
    g.nx = nx; g.ny = ny; g.nz = nz;
    g.sx = b[0]; g.sy = b[2]; g.sz = b[4];
    // MeshStructGenSource constructor (:33-48)
    g.hx = (b[1] - b[0]) / (double) nx;
    g.hy = (b[3] - b[2]) / (double) ny;
    g.hz = (b[5] - b[4]) / (double) nz;
    g.nYZ = ny * nz * (nx + 1);
    g.nXZ = nx * nz * (ny + 1);
    g.nBYZ = ny * nz * 2;
    g.nBXZ = nx * nz * 2;
    return g;
}

int check_dims(int nx, int ny, int nz) {
    CG_RETURN_IF(nx < 1 || ny < 1 || nz < 1, CUPCFD_E_CONFIG_INVALID_VALUE, "generator: dimensions must be >= 1");
    long long nF = (long long) ny * nz * (nx + 1) + (long long) nx * nz * (ny + 1) + (long long) nx * ny * (nz + 1);
    long long nV = (long long) (nx + 1) * (ny + 1) * (nz + 1);
    CG_RETURN_IF(nF >= (1LL << 30) || nV >= (1LL << 31), CUPCFD_E_NOT_IMPLEMENTED, "generator: mesh too large for int32 labels");
    return CUPCFD_E_SUCCESS;
}

int finish(cupcfd_gpu_mesh *m, int rc, cupcfd_gpu_mesh **out) {
    if (rc != CUPCFD_E_SUCCESS) {
        std::string e = cupcfd_gpu_last_error();
        cupcfd_gpu_mesh_destroy(m);
        set_error(e);
        return rc;
    }
    *out = m;
    return CUPCFD_E_SUCCESS;
}

}  // namespace

extern "C" int cupcfd_gpu_mesh_create_structgen(int32_t nx, int32_t ny, int32_t nz, const double bounds[6],
                                                const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) {
    clear_error();
    CG_RETURN_IF(!out, CUPCFD_E_NULL_PTR, "structgen: null output");
    CG_TRY(check_dims(nx, ny, nz));
    const double unit[6] = {0, 1, 0, 1, 0, 1};
    Grid g = make_grid(nx, ny, nz, bounds ? bounds : unit);
    int nC = nx * ny * nz, nF = g.nYZ + g.nXZ + nx * ny * (nz + 1), nB = 2 * (ny * nz + nx * nz + nx * ny);
    cupcfd_gpu_mesh *m;
    CG_TRY(mesh_new(opt, &m));
    cudaStream_t st = m->stream;
    int rc = CUPCFD_E_SUCCESS;
    {
        Pool pool;
        Source s{};
        s.nC = nC; s.nF = nF; s.nB = nB;
        s.c1 = pool.get<int>(nF); s.c2 = pool.get<int>(nF); s.bnd = pool.get<int>(nF);
        s.lam = pool.get<double>(nF); s.area = pool.get<double>(nF);
        s.S = pool.get<double>(3 * (size_t) nF); s.xf = pool.get<double>(3 * (size_t) nF);
        s.cc = pool.get<double>(3 * (size_t) nC); s.vol = pool.get<double>(nC);
        s.xpac = s.xnac = nullptr;  // zero, as addData stores
        if (!s.c1 || !s.c2 || !s.bnd || !s.lam || !s.area || !s.S || !s.xf || !s.cc || !s.vol) {
            set_error("structgen: out of device memory");
            rc = CUPCFD_E_ERROR;
        } else {
            k_structgen_cells<<<grid_for(nC, 256), 256, 0, st>>>(g, nC, s.cc, s.vol);
            g_launches.fetch_add(1);
            k_structgen_faces<<<grid_for(nF, 256), 256, 0, st>>>(g, nF, s.c1, s.c2, s.bnd, s.lam, s.area, s.S, s.xf);
            g_launches.fetch_add(1);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                set_error(std::string("structgen kernels: ") + cudaGetErrorString(e));
                rc = CUPCFD_E_ERROR;
            } else {
                rc = build_mesh_from_source(m, s, opt);
            }
        }
    }
    return finish(m, rc, out);
}

extern "C" int cupcfd_gpu_mesh_create_jittered(int32_t nx, int32_t ny, int32_t nz, double jitter, uint64_t seed,
                                               int32_t permute, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out) {
    clear_error();
    CG_RETURN_IF(!out, CUPCFD_E_NULL_PTR, "jittered: null output");
    CG_TRY(check_dims(nx, ny, nz));
    CG_RETURN_IF(!(jitter >= 0.0 && jitter < 0.5), CUPCFD_E_CONFIG_INVALID_VALUE, "jittered: jitter must be in [0, 0.5)");
    const double unit[6] = {0, 1, 0, 1, 0, 1};
    Grid g = make_grid(nx, ny, nz, unit);
    int nC = nx * ny * nz, nF = g.nYZ + g.nXZ + nx * ny * (nz + 1), nB = 2 * (ny * nz + nx * nz + nx * ny);
    int nV = (nx + 1) * (ny + 1) * (nz + 1);
    std::vector<int> cp(nC), fp(nF);
    if (permute) {
        host_shuffle(cp, seed ^ 0x243F6A8885A308D3ULL);
        host_shuffle(fp, seed ^ 0x13198A2E03707344ULL);
    } else {
        for (int i = 0; i < nC; i++) cp[i] = i;
        for (int i = 0; i < nF; i++) fp[i] = i;
    }
    cupcfd_gpu_mesh *m;
    CG_TRY(mesh_new(opt, &m));
    cudaStream_t st = m->stream;
    int rc = CUPCFD_E_SUCCESS;
    {
        Pool pool;
        double *vc = pool.get<double>(3 * (size_t) nV), *cc = pool.get<double>(3 * (size_t) nC);
        double *vol = pool.get<double>(nC), *lam = pool.get<double>(nF), *area = pool.get<double>(nF);
        double *S = pool.get<double>(3 * (size_t) nF), *xf = pool.get<double>(3 * (size_t) nF), *dvol = pool.get<double>(nF);
        int *f1 = pool.get<int>(nF), *f2 = pool.get<int>(nF), *dcp = pool.get<int>(nC), *dfp = pool.get<int>(nF);
        int *isB = pool.get<int>(nF), *scan = pool.get<int>(nF);
        Source s{};
        s.nC = nC; s.nF = nF; s.nB = nB;
        s.c1 = pool.get<int>(nF); s.c2 = pool.get<int>(nF); s.bnd = pool.get<int>(nF);
        s.lam = pool.get<double>(nF); s.area = pool.get<double>(nF);
        s.S = pool.get<double>(3 * (size_t) nF); s.xf = pool.get<double>(3 * (size_t) nF);
        s.cc = pool.get<double>(3 * (size_t) nC); s.vol = pool.get<double>(nC);
        s.xpac = s.xnac = nullptr;
        size_t tb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tb, isB, scan, nF, st);
        char *tmp = pool.get<char>(tb);
        if (!vc || !cc || !vol || !lam || !area || !S || !xf || !dvol || !f1 || !f2 || !dcp || !dfp || !isB || !scan ||
            !s.c1 || !s.c2 || !s.bnd || !s.lam || !s.area || !s.S || !s.xf || !s.cc || !s.vol || !tmp) {
            set_error("jittered: out of device memory");
            rc = CUPCFD_E_ERROR;
        } else {
            cudaMemcpyAsync(dcp, cp.data(), sizeof(int) * nC, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(dfp, fp.data(), sizeof(int) * nF, cudaMemcpyHostToDevice, st);
            k_jit_verts<<<grid_for(nV, 256), 256, 0, st>>>(g, nV, jitter, (unsigned long long) seed, vc);
            k_jit_centres<<<grid_for(nC, 256), 256, 0, st>>>(g, nC, vc, cc);
            k_jit_faces<<<grid_for(nF, 256), 256, 0, st>>>(g, nF, vc, cc, f1, f2, lam, area, S, xf, dvol);
            k_jit_volumes<<<grid_for(nC, 256), 256, 0, st>>>(g, nC, f1, dvol, vol);
            int n = nF > nC ? nF : nC;
            k_jit_permute<<<grid_for(n, 256), 256, 0, st>>>(nC, nF, dcp, dfp, f1, f2, lam, area, S, xf, cc, vol, s.c1,
                                                            s.c2, isB, s.lam, s.area, s.S, s.xf, s.cc, s.vol);
            cub::DeviceScan::ExclusiveSum(tmp, tb, isB, scan, nF, st);
            k_bnd_ids<<<grid_for(nF, 256), 256, 0, st>>>(nF, isB, scan, s.bnd);
            g_launches.fetch_add(7);
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                set_error(std::string("jittered kernels: ") + cudaGetErrorString(e));
                rc = CUPCFD_E_ERROR;
            } else {
                rc = build_mesh_from_source(m, s, opt);
            }
        }
    }
    return finish(m, rc, out);
}
