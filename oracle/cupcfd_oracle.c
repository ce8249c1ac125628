/*
 * cupcfd_oracle.c - plain-C restatement of the reference's CPU algorithm for
 * the CUP-CFD face-loop path. TEST INFRASTRUCTURE ONLY (see cupcfd_oracle.h):
 * this file is the checker that the CUDA library is compared against; the
 * library never links it.
 *
 * Every floating-point expression keeps the reference's operand order and
 * rounding points (one IEEE operation per C operator, no contraction; the
 * Makefile builds with -ffp-contract=off), so on the same inputs the results
 * are bit-identical to the reference compiled with its Release flags.
 */
#include "cupcfd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* small vector helpers, each one IEEE op per component in reference order    */
/* ------------------------------------------------------------------------- */

/* EuclideanVector::dotProduct (src/geometry/euclidean/implementation/component/EuclideanVector.cpp:83-90):
 * dotP = 0; dotP += a_i*b_i for i = 0..2 */
static double dot3(const double *a, const double *b) {
    double d = 0.0;
    d += a[0] * b[0];
    d += a[1] * b[1];
    d += a[2] * b[2];
    return d;
}

/* EuclideanVector3D::crossProduct (include/geometry/euclidean/implementation/component/EuclideanVector3D.ipp:55-63) */
static void cross3(const double *a, const double *b, double *r) {
    r[0] = (a[1] * b[2]) - (a[2] * b[1]);
    r[1] = (a[2] * b[0]) - (a[0] * b[2]);
    r[2] = (a[0] * b[1]) - (a[1] * b[0]);
}

static void sub3(const double *a, const double *b, double *r) {
    r[0] = a[0] - b[0]; r[1] = a[1] - b[1]; r[2] = a[2] - b[2];
}

/* EuclideanVector::length (EuclideanVector.cpp:92-98): sqrt(dot(v, v)) */
static double len3(const double *v) { return sqrt(dot3(v, v)); }

/* Triangle::heronsFormula (include/geometry/shapes/implementation/component/Triangle.ipp:83-99):
 * lengths ab=|b-a|, ac=|c-a|, bc=|c-b|; s=(ab+ac+bc)/2; sqrt(s*(s-ab)*(s-bc)*(s-ac)) */
static double heron(const double *a, const double *b, const double *c) {
    double t[3];
    sub3(b, a, t); double ab = len3(t);
    sub3(c, a, t); double ac = len3(t);
    sub3(c, b, t); double bc = len3(t);
    double s = (ab + ac + bc) / 2.0;
    return sqrt(s * (s - ab) * (s - bc) * (s - ac));
}

/* ------------------------------------------------------------------------- */
/* structured generator: MeshStructGenSource (src/geometry/mesh/implementation/source/MeshStructGenSource.cpp) */
/* ------------------------------------------------------------------------- */

typedef struct {
    int nx, ny, nz;
    double sminx, sminy, sminz, dsx, dsy, dsz;
    int nFaceYZ, nFaceXZ, nFaceXY, nBndYZ, nBndXZ;
} sg_t;

static void sg_init(sg_t *g, int nx, int ny, int nz, double x0, double x1, double y0, double y1, double z0, double z1) {
    g->nx = nx; g->ny = ny; g->nz = nz;
    g->sminx = x0; g->sminy = y0; g->sminz = z0;
    /* constructor, MeshStructGenSource.cpp:33-48 */
    g->dsx = (x1 - x0) / (double) nx;
    g->dsy = (y1 - y0) / (double) ny;
    g->dsz = (z1 - z0) / (double) nz;
    g->nFaceYZ = ny * nz * (nx + 1);
    g->nFaceXZ = nx * nz * (ny + 1);
    g->nFaceXY = nx * ny * (nz + 1);
    g->nBndYZ = ny * nz * 2;
    g->nBndXZ = nx * nz * 2;
}

void orc_structgen_counts(int nx, int ny, int nz, int *nCells, int *nFaces, int *nBnd, int *nVerts) {
    /* getCellCount/getFaceCount/getBoundaryCount/getVertexCount, MeshStructGenSource.cpp:200-250 */
    *nCells = nx * ny * nz;
    *nFaces = ny * nz * (nx + 1) + nx * nz * (ny + 1) + nx * ny * (nz + 1);
    *nBnd = 2 * (ny * nz + nx * nz + nx * ny);
    *nVerts = (nx + 1) * (ny + 1) * (nz + 1);
}

static int sg_cell(const sg_t *g, int x, int y, int z) { return x + y * g->nx + z * g->nx * g->ny; }
static int sg_vert(const sg_t *g, int x, int y, int z) { return x + y * (g->nx + 1) + z * (g->nx + 1) * (g->ny + 1); }

/* Face label -> orientation (0 YZ, 1 XZ, 2 XY) and the face's integer
 * coordinates in its own label scheme (MeshStructGenSource.cpp:449-500). */
static void sg_face_coords(const sg_t *g, int f, int *kind, int *x, int *y, int *z) {
    if (f < g->nFaceYZ) {
        *kind = 0;
        *x = f % (g->nx + 1); *y = (f / (g->nx + 1)) % g->ny; *z = (f / ((g->nx + 1) * g->ny)) % g->nz;
    } else if (f < g->nFaceYZ + g->nFaceXZ) {
        int l = f - g->nFaceYZ;
        *kind = 1;
        *x = l % g->nx; *y = (l / g->nx) % (g->ny + 1); *z = (l / (g->nx * (g->ny + 1))) % g->nz;
    } else {
        int l = f - g->nFaceYZ - g->nFaceXZ;
        *kind = 2;
        *x = l % g->nx; *y = (l / g->nx) % g->ny; *z = (l / (g->nx * g->ny)) % (g->nz + 1);
    }
}

/* getFaceIsBoundary / getFaceCell1Labels / getFaceCell2Labels / getFaceBoundaryLabels
 * (MeshStructGenSource.cpp:449-822): cell1 is the low-side cell (or the only
 * cell), cell2 the high-side cell or -1. */
static void sg_face_conn(const sg_t *g, int f, int *c1, int *c2, int *bl) {
    int k, x, y, z;
    sg_face_coords(g, f, &k, &x, &y, &z);
    if (k == 0) {
        int hi = (x == g->nx), lo = (x == 0);
        *c1 = sg_cell(g, lo ? x : x - 1, y, z);
        *c2 = (lo || hi) ? -1 : sg_cell(g, x, y, z);
        *bl = lo ? (0 + y * 2 + z * 2 * g->ny) : hi ? (1 + y * 2 + z * 2 * g->ny) : -1;
    } else if (k == 1) {
        int hi = (y == g->ny), lo = (y == 0);
        *c1 = sg_cell(g, x, lo ? y : y - 1, z);
        *c2 = (lo || hi) ? -1 : sg_cell(g, x, y, z);
        *bl = lo ? (g->nBndYZ + x + 0 * g->nx + z * g->nx * 2)
            : hi ? (g->nBndYZ + x + 1 * g->nx + z * g->nx * 2) : -1;
    } else {
        int hi = (z == g->nz), lo = (z == 0);
        *c1 = sg_cell(g, x, y, lo ? z : z - 1);
        *c2 = (lo || hi) ? -1 : sg_cell(g, x, y, z);
        *bl = lo ? (g->nBndYZ + g->nBndXZ + x + y * g->nx + 0 * g->nx * g->ny)
            : hi ? (g->nBndYZ + g->nBndXZ + x + y * g->nx + 1 * g->nx * g->ny) : -1;
    }
}

/* getFaceVerticesLabelsCSR (MeshStructGenSource.cpp:980-1084): four vertex
 * labels in edge order starting at the face's own nodal coordinate. */
static void sg_face_verts(const sg_t *g, int f, int *v) {
    int k, x, y, z;
    sg_face_coords(g, f, &k, &x, &y, &z);
    if (k == 0) {
        v[0] = sg_vert(g, x, y, z); v[1] = sg_vert(g, x, y + 1, z);
        v[2] = sg_vert(g, x, y + 1, z + 1); v[3] = sg_vert(g, x, y, z + 1);
    } else if (k == 1) {
        v[0] = sg_vert(g, x, y, z); v[1] = sg_vert(g, x + 1, y, z);
        v[2] = sg_vert(g, x + 1, y, z + 1); v[3] = sg_vert(g, x, y, z + 1);
    } else {
        v[0] = sg_vert(g, x, y, z); v[1] = sg_vert(g, x + 1, y, z);
        v[2] = sg_vert(g, x + 1, y + 1, z); v[3] = sg_vert(g, x, y + 1, z);
    }
}

/* getVertexCoords (MeshStructGenSource.cpp:1086-1112): smin + ds * coord */
static void sg_vert_coords(const sg_t *g, int v, double *p) {
    int x = v % (g->nx + 1), y = (v / (g->nx + 1)) % (g->ny + 1), z = (v / ((g->nx + 1) * (g->ny + 1))) % (g->nz + 1);
    p[0] = g->sminx + (g->dsx * (double) x);
    p[1] = g->sminy + (g->dsy * (double) y);
    p[2] = g->sminz + (g->dsz * (double) z);
}

/* getCellCenter (MeshStructGenSource.cpp:323-354): low + (high - low)/2 per axis */
static void sg_cell_center(const sg_t *g, int c, double *p) {
    int x = c % g->nx, y = (c / g->nx) % g->ny, z = (c / (g->nx * g->ny)) % g->nz;
    double xl = g->sminx + ((double) x * g->dsx), xh = g->sminx + (double) (x + 1) * g->dsx;
    double yl = g->sminy + ((double) y * g->dsy), yh = g->sminy + ((double) (y + 1) * g->dsy);
    double zl = g->sminz + ((double) z * g->dsz), zh = g->sminz + ((double) (z + 1) * g->dsz);
    p[0] = xl + ((xh - xl) / 2.0);
    p[1] = yl + ((yh - yl) / 2.0);
    p[2] = zl + ((zh - zl) / 2.0);
}

/* Polygon3D::computeArea / computeCentroid for a quad
 * (src/geometry/shapes/interface/component/Polygon3D.cpp:31-55): a triangle fan
 * from v0; area = sum of Heron areas; centroid = area-weighted triangle centroids. */
static void quad_area_centroid(double P[4][3], double *area, double *cen) {
    double a1 = heron(P[0], P[1], P[2]);
    double a2 = heron(P[0], P[2], P[3]);
    double A = 0.0;
    A += a1;
    A += a2;
    double c[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < 3; d++) {
        double t1 = ((P[0][d] + P[1][d]) + P[2][d]) / 3.0;   /* Triangle::computeCentroid */
        double t2 = ((P[0][d] + P[2][d]) + P[3][d]) / 3.0;
        c[d] = c[d] + (t1 * a1);
        c[d] = c[d] + (t2 * a2);
        cen[d] = c[d] / A;
    }
    *area = A;
}

/* getFaceNormal (MeshStructGenSource.cpp:887-946) with isVertexOrderClockwise
 * (Polygon3D.cpp:93-119) and EuclideanPlane3D::calculateNormal
 * (src/geometry/euclidean/implementation/component/EuclideanPlane3D.cpp:203-210):
 * n = (v1-v0)x(v2-v0) when the vertices are clockwise seen from cell1's
 * centre, else (v1-v2)x(v0-v2). */
static void quad_normal_from(double P[4][3], const double *obs, double *n) {
    double u[3], v[3], nn[3], o[3];
    sub3(P[1], P[0], u); sub3(P[2], P[0], v); cross3(u, v, nn);
    sub3(obs, P[0], o);
    if (dot3(nn, o) < 0.0) {
        n[0] = nn[0]; n[1] = nn[1]; n[2] = nn[2];
    } else {
        sub3(P[1], P[2], u); sub3(P[0], P[2], v); cross3(u, v, n);
    }
}

int orc_structgen_build(int nx, int ny, int nz,
                        double xmin, double xmax, double ymin, double ymax, double zmin, double zmax,
                        int *faceCell1, int *faceCell2, int *faceBnd,
                        double *faceLambda, double *faceNorm, double *faceCenter, double *faceArea,
                        double *cellCenter, double *cellVolume, int *faceVert, double *vertCoords) {
    if (nx < 1 || ny < 1 || nz < 1) return ORC_E_ERROR;
    sg_t g;
    sg_init(&g, nx, ny, nz, xmin, xmax, ymin, ymax, zmin, zmax);
    int nC, nF, nB, nV;
    orc_structgen_counts(nx, ny, nz, &nC, &nF, &nB, &nV);
    for (int c = 0; c < nC; c++) {
        double p[3];
        sg_cell_center(&g, c, p);
        cellCenter[3 * c] = p[0]; cellCenter[3 * c + 1] = p[1]; cellCenter[3 * c + 2] = p[2];
        /* The reference builds a Hexahedron from centre +- ds/2 and sums five
         * tetrahedra (MeshStructGenSource.cpp:278-322, Hexahedron.ipp:135-139).
         * For this axis-aligned box the restatement uses the box volume
         * directly; the two agree to 2e-14 relative, the rounding of the Heron
         * sum (checked against the reference build in
         * tests/test_oracle_vs_reference.py). */
        int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        double xl = g.sminx + ((double) x * g.dsx), xh = g.sminx + (double) (x + 1) * g.dsx;
        double yl = g.sminy + ((double) y * g.dsy), yh = g.sminy + ((double) (y + 1) * g.dsy);
        double zl = g.sminz + ((double) z * g.dsz), zh = g.sminz + ((double) (z + 1) * g.dsz);
        cellVolume[c] = ((xh - xl) * (yh - yl)) * (zh - zl);
    }
    for (int f = 0; f < nF; f++) {
        int c1, c2, bl, vl[4];
        sg_face_conn(&g, f, &c1, &c2, &bl);
        faceCell1[f] = c1; faceCell2[f] = c2; faceBnd[f] = bl;
        faceLambda[f] = (bl >= 0) ? -1.0 : 0.5;             /* getFaceLambda, :824-850 */
        sg_face_verts(&g, f, vl);
        double P[4][3];
        for (int k = 0; k < 4; k++) {
            sg_vert_coords(&g, vl[k], P[k]);
            if (faceVert) faceVert[4 * f + k] = vl[k];
        }
        double a, cen[3], n[3];
        quad_area_centroid(P, &a, cen);                     /* getFaceArea :852, getFaceCenter :947 */
        quad_normal_from(P, &cellCenter[3 * c1], n);        /* getFaceNormal :887 */
        faceArea[f] = a;
        for (int d = 0; d < 3; d++) { faceCenter[3 * f + d] = cen[d]; faceNorm[3 * f + d] = n[d]; }
    }
    if (vertCoords)
        for (int v = 0; v < nV; v++) sg_vert_coords(&g, v, &vertCoords[3 * v]);
    return ORC_E_SUCCESS;
}

/* getCellFaceLabels (MeshStructGenSource.cpp:356-447): per cell, in the order
 * XLow, XHigh, YLow, YHigh, ZLow, ZHigh. */
int orc_structgen_cell_face_labels(int nx, int ny, int nz, int *xadj, int *adj) {
    sg_t g;
    sg_init(&g, nx, ny, nz, 0, 1, 0, 1, 0, 1);
    int nC = nx * ny * nz;
    for (int c = 0; c < nC; c++) {
        int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        int *o = &adj[6 * c];
        xadj[c] = 6 * c;
        o[0] = x + y * (nx + 1) + z * (nx + 1) * ny;
        o[1] = (x + 1) + y * (nx + 1) + z * (nx + 1) * ny;
        o[2] = g.nFaceYZ + x + y * nx + z * nx * (ny + 1);
        o[3] = g.nFaceYZ + x + (y + 1) * nx + z * nx * (ny + 1);
        o[4] = g.nFaceYZ + g.nFaceXZ + x + y * nx + z * nx * ny;
        o[5] = g.nFaceYZ + g.nFaceXZ + x + y * nx + (z + 1) * nx * ny;
    }
    xadj[nC] = 6 * nC;
    return ORC_E_SUCCESS;
}

/* ------------------------------------------------------------------------- */
/* jittered + permuted hex mesh                                               */
/* ------------------------------------------------------------------------- */
/* The reference has no such generator: its unstructured meshes come from
 * HDF5 files (MeshHDF5Source.cpp) whose geometry arrays are precomputed. This
 * generator defines that geometry as follows, and the CUDA library's
 * generator states the same definition:
 *   - vertices on the structured grid; every vertex not on the domain
 *     boundary is displaced by U[-jitter*h, +jitter*h] per axis (h = spacing
 *     on that axis) from a splitmix64 stream keyed by (seed, vertex, axis);
 *   - face area vector S = 0.5 * (v2 - v0) x (v3 - v1), oriented away from
 *     cell1; area = |S|; face centre = mean of its 4 vertices;
 *   - cell centre = mean of its 8 vertices; volume = sum over its 6 faces of
 *     (x_f . S_f,outward) / 3;
 *   - lambda (weight of cell2) = ((x_f - x_1) . S) / ((x_2 - x_1) . S) on
 *     interior faces, -1 on boundary faces;
 *   - with permute != 0, cell and face labels are shuffled by seeded
 *     Fisher-Yates permutations (cellPerm[old] = new, facePerm[old] = new)
 *     and boundary ids are numbered in ascending new face label.
 */
static unsigned long long splitmix64(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
/* uniform in [-1, 1) from the top 53 bits */
static double hash_unit(unsigned long long seed, unsigned long long key) {
    unsigned long long r = splitmix64(seed ^ splitmix64(key));
    return ((double) (r >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
}

static void shuffle(int *perm, int n, unsigned long long seed) {
    for (int i = 0; i < n; i++) perm[i] = i;
    unsigned long long s = seed;
    for (int i = n - 1; i > 0; i--) {
        s = splitmix64(s);
        int j = (int) (s % (unsigned long long) (i + 1));
        int t = perm[i]; perm[i] = perm[j]; perm[j] = t;
    }
}

int orc_jitter_build(int nx, int ny, int nz, double jitter, unsigned long long seed, int permute,
                     int *faceCell1, int *faceCell2, int *faceBnd,
                     double *faceLambda, double *faceNorm, double *faceCenter, double *faceArea,
                     double *cellCenter, double *cellVolume, int *cellPerm, int *facePerm) {
    if (nx < 1 || ny < 1 || nz < 1) return ORC_E_ERROR;
    sg_t g;
    sg_init(&g, nx, ny, nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0);
    int nC, nF, nB, nV;
    orc_structgen_counts(nx, ny, nz, &nC, &nF, &nB, &nV);
    double *vc = (double *) malloc(sizeof(double) * 3 * (size_t) nV);
    double *cc = (double *) calloc(3 * (size_t) nC, sizeof(double));
    double *cv = (double *) calloc((size_t) nC, sizeof(double));
    double *fS = (double *) malloc(sizeof(double) * 3 * (size_t) nF);
    double *fX = (double *) malloc(sizeof(double) * 3 * (size_t) nF);
    double *fA = (double *) malloc(sizeof(double) * (size_t) nF);
    double *fL = (double *) malloc(sizeof(double) * (size_t) nF);
    int *f1 = (int *) malloc(sizeof(int) * (size_t) nF), *f2 = (int *) malloc(sizeof(int) * (size_t) nF);
    if (!vc || !cc || !cv || !fS || !fX || !fA || !fL || !f1 || !f2) return ORC_E_ERROR;
    double h[3] = {g.dsx, g.dsy, g.dsz};
    for (int v = 0; v < nV; v++) {
        int x = v % (nx + 1), y = (v / (nx + 1)) % (ny + 1), z = v / ((nx + 1) * (ny + 1));
        sg_vert_coords(&g, v, &vc[3 * v]);
        int interior = (x > 0 && x < nx && y > 0 && y < ny && z > 0 && z < nz);
        if (interior)
            for (int d = 0; d < 3; d++)
                vc[3 * v + d] += jitter * h[d] * hash_unit(seed, 3ULL * (unsigned long long) v + (unsigned long long) d);
    }
    /* cell centres: mean of 8 vertices (x fastest, then y, then z) */
    for (int c = 0; c < nC; c++) {
        int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
        double s[3] = {0, 0, 0};
        for (int k = 0; k < 8; k++) {
            int v = sg_vert(&g, x + (k & 1), y + ((k >> 1) & 1), z + ((k >> 2) & 1));
            for (int d = 0; d < 3; d++) s[d] += vc[3 * v + d];
        }
        for (int d = 0; d < 3; d++) cc[3 * c + d] = s[d] / 8.0;
    }
    for (int f = 0; f < nF; f++) {
        int c1, c2, bl, vl[4];
        sg_face_conn(&g, f, &c1, &c2, &bl);
        f1[f] = c1; f2[f] = c2;
        sg_face_verts(&g, f, vl);
        const double *p0 = &vc[3 * vl[0]], *p1 = &vc[3 * vl[1]], *p2 = &vc[3 * vl[2]], *p3 = &vc[3 * vl[3]];
        double d1[3], d2[3], S[3], xf[3], r[3];
        sub3(p2, p0, d1); sub3(p3, p1, d2); cross3(d1, d2, S);
        for (int d = 0; d < 3; d++) { S[d] = 0.5 * S[d]; xf[d] = (((p0[d] + p1[d]) + p2[d]) + p3[d]) / 4.0; }
        sub3(xf, &cc[3 * c1], r);
        if (dot3(S, r) < 0.0) for (int d = 0; d < 3; d++) S[d] = -S[d];
        for (int d = 0; d < 3; d++) { fS[3 * f + d] = S[d]; fX[3 * f + d] = xf[d]; }
        fA[f] = len3(S);
        double dv = dot3(xf, S) / 3.0;
        cv[c1] += dv;
        if (c2 >= 0) {
            cv[c2] -= dv;
            double a[3], b[3];
            sub3(xf, &cc[3 * c1], a); sub3(&cc[3 * c2], &cc[3 * c1], b);
            fL[f] = dot3(a, S) / dot3(b, S);
        } else {
            fL[f] = -1.0;
        }
    }
    /* permutations */
    int *cp = cellPerm, *fp = facePerm;
    if (permute) {
        shuffle(cp, nC, seed ^ 0x243F6A8885A308D3ULL);
        shuffle(fp, nF, seed ^ 0x13198A2E03707344ULL);
    } else {
        for (int i = 0; i < nC; i++) cp[i] = i;
        for (int i = 0; i < nF; i++) fp[i] = i;
    }
    for (int c = 0; c < nC; c++) {
        int n = cp[c];
        for (int d = 0; d < 3; d++) cellCenter[3 * n + d] = cc[3 * c + d];
        cellVolume[n] = cv[c];
    }
    for (int f = 0; f < nF; f++) {
        int n = fp[f];
        faceCell1[n] = cp[f1[f]];
        faceCell2[n] = f2[f] >= 0 ? cp[f2[f]] : -1;
        faceLambda[n] = fL[f];
        faceArea[n] = fA[f];
        for (int d = 0; d < 3; d++) { faceNorm[3 * n + d] = fS[3 * f + d]; faceCenter[3 * n + d] = fX[3 * f + d]; }
    }
    int b = 0;
    for (int n = 0; n < nF; n++) faceBnd[n] = (faceCell2[n] < 0) ? b++ : -1;
    free(vc); free(cc); free(cv); free(fS); free(fX); free(fA); free(fL); free(f1); free(f2);
    return (b == nB) ? ORC_E_SUCCESS : ORC_E_ERROR;
}

/* ------------------------------------------------------------------------- */
/* cell -> face CSR: CupCfdSoAMesh::updateCellFaceMap (CupCfdSoAMesh.cpp:549-668)
 * Offsets are the running sum of per-cell face counts; faces are placed in
 * ascending face id into the first free slot of cell1 then cell2, and each
 * cell's list is finally sorted ascending (merge_sort, :613-621).            */
/* ------------------------------------------------------------------------- */
static int cmp_int(const void *a, const void *b) {
    int x = *(const int *) a, y = *(const int *) b;
    return (x > y) - (x < y);
}

int orc_cell_face_csr(int nCells, int nFaces, const int *faceCell1, const int *faceCell2, int *xadj, int *adj) {
    int *cnt = (int *) calloc((size_t) nCells + 1, sizeof(int));
    if (!cnt) return ORC_E_ERROR;
    for (int f = 0; f < nFaces; f++) {
        int a = faceCell1[f], b = faceCell2[f];
        if (a < 0 || a >= nCells || b >= nCells) { free(cnt); return ORC_E_INVALID_INDEX; }
        cnt[a]++;
        if (b > -1) cnt[b]++;
    }
    int ptr = 0;
    for (int c = 0; c < nCells; c++) { xadj[c] = ptr; ptr += cnt[c]; }
    xadj[nCells] = ptr;
    for (int k = 0; k < ptr; k++) adj[k] = -1;
    for (int f = 0; f < nFaces; f++) {
        int cs[2] = {faceCell1[f], faceCell2[f]};
        for (int r = 0; r < 2; r++) {
            if (cs[r] < 0) continue;
            for (int j = xadj[cs[r]]; j < xadj[cs[r] + 1]; j++)
                if (adj[j] == -1) { adj[j] = f; break; }
        }
    }
    for (int c = 0; c < nCells; c++)
        qsort(&adj[xadj[c]], (size_t) (xadj[c + 1] - xadj[c]), sizeof(int), cmp_int);
    free(cnt);
    return ORC_E_SUCCESS;
}

/* ------------------------------------------------------------------------- */
/* GradientPhiGaussDolfyn (include/fvm/implementation/component/GradientKernels.ipp:38-136) */
/* ------------------------------------------------------------------------- */
int orc_gradient_phi_gauss(const orc_mesh *m, int nGradient,
                           const double *phi, int nPhi, const double *phiB, int nPhiB,
                           double *g, int nG, double *go, int nGo) {
    /* index checks of the reference's DEBUG build (:90-95, :107-111) */
    for (int f = 0; f < m->nFaces; f++) {
        int ip = m->faceCell1[f], in = m->faceCell2[f], ib = m->faceBnd[f];
        if (ib > -1) { if (ib >= nPhiB || ip >= nPhi) return ORC_E_INVALID_INDEX; }
        else if (ip >= nPhi || in >= nPhi) return ORC_E_INVALID_INDEX;
    }
    if (nG < m->nCells) return ORC_E_INVALID_INDEX;
    for (int i = 0; i < 3 * nGo; i++) go[i] = 0.0;                        /* :57-61 */
    for (int it = 0; it < nGradient; it++) {
        for (int i = 0; i < 3 * nG; i++) g[i] = 0.0;                      /* :66-70 */
        for (int f = 0; f < m->nFaces; f++) {                              /* :73-116 */
            int ip = m->faceCell1[f];
            int in = m->faceCell2[f];
            const double *S = &m->faceNorm[3 * f];
            double phiFace;
            if (!(m->faceBnd[f] > -1)) {
                double facn = m->faceLambda[f];
                double facp = 1.0 - facn;
                double xac[3], gac[3], corr[3];
                for (int d = 0; d < 3; d++) {
                    xac[d] = (m->cellCenter[3 * in + d] * facn) + (m->cellCenter[3 * ip + d] * facp);
                    gac[d] = (go[3 * in + d] * facn) + (go[3 * ip + d] * facp);
                }
                phiFace = (phi[in] * facn) + (phi[ip] * facp);
                for (int d = 0; d < 3; d++) corr[d] = m->faceCenter[3 * f + d] - xac[d];
                phiFace += dot3(gac, corr);
                for (int d = 0; d < 3; d++) g[3 * ip + d] += phiFace * S[d];    /* :102 */
                for (int d = 0; d < 3; d++) g[3 * in + d] += phiFace * S[d];    /* :103, same sign (H1) */
            } else {
                phiFace = phiB[m->faceBnd[f]];
                for (int d = 0; d < 3; d++) g[3 * ip + d] += phiFace * S[d];
            }
        }
        for (int i = 0; i < m->nCells; i++) {                              /* :122-126 */
            double fact = 1.0 / m->cellVolume[i];
            for (int d = 0; d < 3; d++) g[3 * i + d] *= fact;
        }
        for (int i = 0; i < 3 * nGo; i++) go[i] = g[i];                     /* :129-131 */
    }
    return ORC_E_SUCCESS;
}

/* ------------------------------------------------------------------------- */
/* FluxMassDolfynFaceLoop (include/fvm/implementation/component/MassKernels.ipp:36-309) */
/* ------------------------------------------------------------------------- */
int orc_flux_mass_face_loop(const orc_mesh *m,
                            const double *dudx, const double *dvdx, const double *dwdx, const double *dpdx,
                            const double *den, double *denB, const double *u, const double *v, const double *w,
                            double *massFlux, const double *p, const double *ar, double *su, double *rface,
                            double small, int *icinl, int *icout, int *icsym, int *icwal,
                            int solveTurbEnergy, int solveTurbDiss, int solveVisc, int solveEnthalpy,
                            const double *teC, double *teB, const double *edC, double *edB,
                            const double *visC, double *visB, const double *tC, double *tB) {
    for (int i = 0; i < m->nFaces; i++) {
        int ip = m->faceCell1[i], in = m->faceCell2[i];
        const double *S = &m->faceNorm[3 * i];
        if (!(m->faceBnd[i] > -1)) {
            const double *cP = &m->cellCenter[3 * ip], *cN = &m->cellCenter[3 * in];
            double facn = m->faceLambda[i];
            double facp = 1.0 - facn;
            double duac[3], dvac[3], dwac[3], xac[3], delta[3];
            for (int d = 0; d < 3; d++) {
                duac[d] = dudx[3 * in + d] * facn + dudx[3 * ip + d] * facp;       /* :142-144 */
                dvac[d] = dvdx[3 * in + d] * facn + dvdx[3 * ip + d] * facp;
                dwac[d] = dwdx[3 * in + d] * facn + dwdx[3 * ip + d] * facp;
            }
            double denf = den[in] * facn + den[ip] * facp;                         /* :146 */
            for (int d = 0; d < 3; d++) {
                xac[d] = cN[d] * facn + cP[d] * facp;                               /* :147 */
                delta[d] = m->faceCenter[3 * i + d] - xac[d];                       /* :148-149 */
            }
            double uFace = u[in] * facn + u[ip] * facp + dot3(duac, delta);         /* :151-153 */
            double vFace = v[in] * facn + v[ip] * facp + dot3(dvac, delta);
            double wFace = w[in] * facn + w[ip] * facp + dot3(dwac, delta);
            massFlux[i] = denf * (uFace * S[0] + vFace * S[1] + wFace * S[2]);      /* :155-157 */
            double xnorm[3] = {S[0], S[1], S[2]};                                   /* :159-160 normalise */
            double len = len3(xnorm);
            if (len != 0.0) {
                double s = 1.0 / len;
                for (int d = 0; d < 3; d++) xnorm[d] *= s;
            }
            const double *xpac = &m->faceXpac[3 * i], *xnac = &m->faceXnac[3 * i];
            double delp[3], deln[3], xpn[3], xpn2[3];
            sub3(xpac, cP, delp);
            double pip = p[ip] + dot3(&dpdx[3 * ip], delp);                          /* :165-166 */
            sub3(xpac, cN, deln);
            double pin = p[in] + dot3(&dpdx[3 * ip], deln);                          /* :168-169, dpdx[ip] (H7) */
            sub3(xnac, xpac, xpn);
            sub3(cN, cP, xpn2);
            double apv1 = den[ip] * ar[ip];
            double apv2 = den[in] * ar[in];
            double apv = apv2 * facn + apv1 * facp;
            double factv = m->cellVolume[in] * facn + m->cellVolume[ip] * facp;
            apv *= m->faceArea[i] * factv / dot3(xpn2, xnorm);                     /* :179 */
            double dpx = (dpdx[3 * in + 0] * facn + dpdx[3 * ip + 0] * facp) * xpn[0];
            double dpy = (dpdx[3 * in + 1] * facn + dpdx[3 * ip + 1] * facp) * xpn[1];
            double dpz = (dpdx[3 * in + 2] * facn + dpdx[3 * ip + 2] * facp) * xpn[2];
            double fact = apv;
            rface[2 * i] = -fact;                                                   /* :192-193 */
            rface[2 * i + 1] = -fact;
            massFlux[i] = massFlux[i] - fact * ((pin - pip) - dpx - dpy - dpz);    /* :195 */
        } else {
            int ib = m->faceBnd[i];
            int ir = m->bndRegion[ib];
            int it = m->regionType[ir];
            if (it == ORC_RTYPE_INLET) {                                            /* :248-259 */
                *icinl = *icinl + 1;
                double dens = m->regionDen[ir];
                massFlux[i] = dens * dot3(&m->regionUVW[3 * ir], S);
                su[ip] = su[ip] - massFlux[i];
            } else if (it == ORC_RTYPE_OUTLET) {                                    /* :260-296 */
                *icout = *icout + 1;
                double uF = u[ip], vF = v[ip], wF = w[ip];
                double denf = den[ip];
                denB[ib] = denf;
                massFlux[i] = denf * (uF * S[0] + vF * S[1] + wF * S[2]);
                if (massFlux[i] < 0.0) {
                    massFlux[i] = small;
                    if (solveTurbEnergy) teB[ib] = teC[ip];
                    if (solveTurbDiss) edB[ib] = edC[ip];
                    if (solveVisc) visB[ib] = visC[ip];
                    if (solveEnthalpy) tB[ib] = tC[ip];
                }
            } else if (it == ORC_RTYPE_SYMP) {                                      /* :297-300 */
                *icsym = *icsym + 1;
                massFlux[i] = 0.0;
            } else if (it == ORC_RTYPE_WALL) {                                      /* :301-304 */
                *icwal = *icwal + 1;
                massFlux[i] = 0.0;
            }
        }
    }
    return ORC_E_SUCCESS;
}

/* ------------------------------------------------------------------------- */
/* plain mass flux m_f = rho_f (u_f . S_f) and the adjoints (no reference counterpart) */
/* ------------------------------------------------------------------------- */
/* Equals FluxMassDolfynFaceLoop with zero velocity gradients, zero pressure
 * and zero pressure gradient on interior faces; boundary faces are left
 * unchanged, as the reference does for RTYPE_DEFAULT regions. */
int orc_mass_plain_forward(const orc_mesh *m, const double *den, const double *u, const double *v, const double *w,
                           double *massFlux) {
    for (int i = 0; i < m->nFaces; i++) {
        if (m->faceBnd[i] > -1) continue;
        int ip = m->faceCell1[i], in = m->faceCell2[i];
        const double *S = &m->faceNorm[3 * i];
        double facn = m->faceLambda[i], facp = 1.0 - facn;
        double denf = den[in] * facn + den[ip] * facp;
        double uF = u[in] * facn + u[ip] * facp;
        double vF = v[in] * facn + v[ip] * facp;
        double wF = w[in] * facn + w[ip] * facp;
        massFlux[i] = denf * (uF * S[0] + vF * S[1] + wF * S[2]);
    }
    return ORC_E_SUCCESS;
}

int orc_mass_plain_adjoint(const orc_mesh *m, const double *den, const double *u, const double *v, const double *w,
                           const double *mbar, double *denbar, double *ubar, double *vbar, double *wbar) {
    for (int c = 0; c < m->nCells; c++) { denbar[c] = 0.0; ubar[c] = 0.0; vbar[c] = 0.0; wbar[c] = 0.0; }
    for (int i = 0; i < m->nFaces; i++) {
        if (m->faceBnd[i] > -1) continue;
        int ip = m->faceCell1[i], in = m->faceCell2[i];
        const double *S = &m->faceNorm[3 * i];
        double facn = m->faceLambda[i], facp = 1.0 - facn;
        double denf = den[in] * facn + den[ip] * facp;
        double uF = u[in] * facn + u[ip] * facp;
        double vF = v[in] * facn + v[ip] * facp;
        double wF = w[in] * facn + w[ip] * facp;
        double flux = uF * S[0] + vF * S[1] + wF * S[2];
        double gr = mbar[i] * flux;          /* dL/d rho_f */
        double gu = mbar[i] * denf;          /* dL/d (u_f . S) */
        denbar[ip] += facp * gr; denbar[in] += facn * gr;
        ubar[ip] += facp * gu * S[0]; ubar[in] += facn * gu * S[0];
        vbar[ip] += facp * gu * S[1]; vbar[in] += facn * gu * S[1];
        wbar[ip] += facp * gu * S[2]; wbar[in] += facn * gu * S[2];
    }
    return ORC_E_SUCCESS;
}

/* Adjoint of GradientPhiGaussDolfyn with nGradient = 1 (the correction term
 * is then identically zero, GradientKernels.ipp:57-61): dPhidx_c =
 * (1/V_c) sum_f phi_f S_f with the same sign for both cells, so
 * dL/dphi_f = sum over the face's cells c of (gbar_c / V_c) . S_f, and
 * phi_f = lambda phi_N + (1 - lambda) phi_P spreads it back. */
int orc_gradient_adjoint(const orc_mesh *m, const double *gbar, double *phibar, double *phibBar) {
    for (int c = 0; c < m->nCells; c++) phibar[c] = 0.0;
    for (int b = 0; b < m->nBnd; b++) phibBar[b] = 0.0;
    for (int i = 0; i < m->nFaces; i++) {
        int ip = m->faceCell1[i], in = m->faceCell2[i];
        const double *S = &m->faceNorm[3 * i];
        double fP = 1.0 / m->cellVolume[ip];
        double hP = (gbar[3 * ip] * S[0] + gbar[3 * ip + 1] * S[1] + gbar[3 * ip + 2] * S[2]) * fP;
        if (m->faceBnd[i] > -1) {
            phibBar[m->faceBnd[i]] += hP;
        } else {
            double fN = 1.0 / m->cellVolume[in];
            double hN = (gbar[3 * in] * S[0] + gbar[3 * in + 1] * S[1] + gbar[3 * in + 2] * S[2]) * fN;
            double pf = hP + hN;
            double facn = m->faceLambda[i], facp = 1.0 - facn;
            phibar[ip] += facp * pf;
            phibar[in] += facn * pf;
        }
    }
    return ORC_E_SUCCESS;
}

/* ------------------------------------------------------------------------ */
/* Boundary / region loops (MassKernels.ipp:311-554).                       */
/* The reference walks boundaries ib = 0 .. nBnd-1 and reaches each one's   */
/* face through getBoundaryFaceID; here that map is faceBnd inverted.        */
/* ------------------------------------------------------------------------ */
static int *orc_boundary_faces(const orc_mesh *m) {
    int *bf = (int *) malloc(sizeof(int) * (size_t) (m->nBnd > 0 ? m->nBnd : 1));
    if (!bf) return NULL;
    for (int b = 0; b < m->nBnd; b++) bf[b] = -1;
    for (int f = 0; f < m->nFaces; f++)
        if (m->faceBnd[f] > -1) bf[m->faceBnd[f]] = f;
    return bf;
}

static int orc_btype(const orc_mesh *m, int ib) { return m->regionType[m->bndRegion[ib]]; }

/* FluxMassDolfynBoundaryLoop1 (MassKernels.ipp:311-336): inlet mass inflow. */
int orc_boundary_loop1(const orc_mesh *m, const double *massFlux, double *flowin) {
    int *bf = orc_boundary_faces(m);
    if (!bf) return ORC_E_ERROR;
    *flowin = 0.0;
    for (int ib = 0; ib < m->nBnd; ib++)
        if (orc_btype(m, ib) == ORC_RTYPE_INLET) *flowin = *flowin + massFlux[bf[ib]];
    free(bf);
    return ORC_E_SUCCESS;
}

/* FluxMassDolfynBoundaryLoop2 (MassKernels.ipp:338-368): outlet outflow, in
 * total and per region (flowRegion accumulates onto its input). */
int orc_boundary_loop2(const orc_mesh *m, const double *massFlux, double *flowRegion, double *flowout) {
    int *bf = orc_boundary_faces(m);
    if (!bf) return ORC_E_ERROR;
    *flowout = 0.0;
    for (int ib = 0; ib < m->nBnd; ib++) {
        int ir = m->bndRegion[ib];
        if (m->regionType[ir] == ORC_RTYPE_OUTLET) {
            int i = bf[ib];
            *flowout = *flowout + massFlux[i];
            flowRegion[ir] = flowRegion[ir] + massFlux[i];
        }
    }
    free(bf);
    return ORC_E_SUCCESS;
}

/* FluxMassDolfynBoundaryLoop3 (MassKernels.ipp:371-393): outlet area and the
 * area rate -flowin / areaout. */
int orc_boundary_loop3(const orc_mesh *m, double flowin, double *ratearea) {
    int *bf = orc_boundary_faces(m);
    if (!bf) return ORC_E_ERROR;
    double areaout = 0.0;
    for (int ib = 0; ib < m->nBnd; ib++)
        if (orc_btype(m, ib) == ORC_RTYPE_OUTLET) areaout = areaout + m->faceArea[bf[ib]];
    *ratearea = -flowin / areaout;
    free(bf);
    return ORC_E_SUCCESS;
}

/* FluxMassDolfynBoundaryLoop4 (MassKernels.ipp:395-454): outlet mass flux
 * from the area rate, and the outlet velocities along the unit normal. */
int orc_boundary_loop4(const orc_mesh *m, const double *splvl, double *massFlux, double *uB, double *vB, double *wB,
                       const double *denB, double ratearea, double *flowout) {
    int *bf = orc_boundary_faces(m);
    if (!bf) return ORC_E_ERROR;
    *flowout = 0.0;
    for (int ib = 0; ib < m->nBnd; ib++) {
        int ir = m->bndRegion[ib];
        if (m->regionType[ir] != ORC_RTYPE_OUTLET) continue;
        int i = bf[ib];
        double split = splvl[ir];
        double area = m->faceArea[i];
        massFlux[i] = ratearea * area * split;
        double faceFlux = massFlux[i] / denB[ib] / area;
        /* EuclideanVector::normalise (EuclideanVector.cpp:100-109): length is
         * sqrt of the dot product accumulated from 0 (EuclideanVector.cpp:83-98) */
        double x[3] = {m->faceNorm[3 * i], m->faceNorm[3 * i + 1], m->faceNorm[3 * i + 2]};
        double dot = 0.0;
        for (int d = 0; d < 3; d++) dot += x[d] * x[d];
        double scalar = sqrt(dot);
        if (scalar != 0.0) {
            scalar = 1.0 / scalar;
            for (int d = 0; d < 3; d++) x[d] *= scalar;
        }
        uB[ib] = faceFlux * x[0];
        vB[ib] = faceFlux * x[1];
        wB[ib] = faceFlux * x[2];
        *flowout = *flowout + massFlux[i];
    }
    free(bf);
    return ORC_E_SUCCESS;
}

/* FluxMassDolfynBoundaryLoop5 (MassKernels.ipp:457-521): outlet mass flux
 * scaled by its region's factor, accumulated onto *flowout2 (not reset),
 * optional velocity scaling, and su[cell1] -= massFlux, boundary by boundary. */
int orc_boundary_loop5(const orc_mesh *m, double *massFlux, double *su, double *uB, double *vB, double *wB, double fact,
                       int solveU, int solveV, int solveW, const double *flowFact, double *flowout2) {
    int *bf = orc_boundary_faces(m);
    if (!bf) return ORC_E_ERROR;
    for (int ib = 0; ib < m->nBnd; ib++) {
        int ir = m->bndRegion[ib];
        if (m->regionType[ir] != ORC_RTYPE_OUTLET) continue;
        int i = bf[ib];
        massFlux[i] = massFlux[i] * flowFact[ir];
        *flowout2 = *flowout2 + massFlux[i];
        if (solveU) uB[ib] = uB[ib] * fact;
        if (solveV) vB[ib] = vB[ib] * fact;
        if (solveW) wB[ib] = wB[ib] * fact;
        int ip = m->faceCell1[i];
        su[ip] = su[ip] - massFlux[i];
    }
    free(bf);
    return ORC_E_SUCCESS;
}

/* FluxMassDolfynRegionLoop (MassKernels.ipp:523-554): per-region outflow
 * factor -(split * flowIn) / flowRegion on outlets, 0 elsewhere. */
int orc_region_loop(const orc_mesh *m, const double *splvl, double *flowFact, const double *flowRegion, double flowIn) {
    for (int ir = 0; ir < m->nRegions; ir++) {
        if (m->regionType[ir] == ORC_RTYPE_OUTLET) {
            double split = splvl[ir];
            flowFact[ir] = -(split * flowIn) / flowRegion[ir];
        } else {
            flowFact[ir] = 0.0;
        }
    }
    return ORC_E_SUCCESS;
}

/* ------------------------------------------------------------------------- */
/* Momentum face loop (include/fvm/implementation/component/UVWKernels.ipp)  */
/* ------------------------------------------------------------------------- */

/* std::min / std::max as <algorithm> defines them: min(a,b) = b < a ? b : a,
 * max(a,b) = a < b ? b : a (the first argument wins ties and NaN compares). */
static double std_min(double a, double b) { return (b < a) ? b : a; }
static double std_max(double a, double b) { return (a < b) ? b : a; }

/* EuclideanVector::normalise (EuclideanVector.cpp:100-109) */
static void normalise3(double *x) {
    double len = sqrt(dot3(x, x));
    if (len != 0.0) {
        double sc = 1.0 / len;
        x[0] *= sc; x[1] *= sc; x[2] *= sc;
    }
}

/* FluxUVWDolfynFaceLoop1 (UVWKernels.ipp:38-515), face by face in label
 * order. uFace/vFace/wFace and visFace are declared outside the face loop
 * (UVWKernels.ipp:74-75) and carry from one face to the next: interior faces
 * read the uFace the last inlet or outlet face set (the interpolation that
 * would set it is commented out, UVWKernels.ipp:165-168, read at :171), symmetry faces read
 * the visFace the last interior, inlet or outlet face set. The reference
 * leaves them uninitialised; here they start at 0. rlencos[nFaces] and
 * bndDist[nBnd] stand for getFaceRLencos / getBoundaryDistance (NULL reads 0,
 * as every MeshSource-built mesh holds, UnstructuredMeshInterface.ipp:1809-1810,
 * MeshStructGenSource.cpp:1251-1258); shear[3*nBnd] receives setBoundaryShear
 * (wall faces only). Vector fields are xyz-interleaved [3*nCells]. */
int orc_uvw_face_loop1(const orc_mesh *m, const double *rlencos, const double *bndDist, double gammaBlend, double small,
                       const double *u, const double *v, const double *w, double *uB, double *vB, double *wB,
                       const double *visC, const double *visB, double *massFlux,
                       const double *dudx, const double *dvdx, const double *dwdx, double *rFace,
                       double *su, double *sv, double *sw, double *au, double *av, double *aw, double *shear) {
    double uFace = 0.0, vFace = 0.0, wFace = 0.0, visFace = 0.0;
    for (int i = 0; i < m->nFaces; i++) {
        int ip = m->faceCell1[i];
        const double *S = m->faceNorm + 3 * i;
        double rl = rlencos ? rlencos[i] : 0.0;
        if (m->faceBnd[i] < 0) {
            int in = m->faceCell2[i];
            double facn = m->faceLambda[i];
            double facp = 1.0 - facn;
            double du[3], dv[3], dw[3], xpn[3];
            for (int d = 0; d < 3; d++) {
                du[d] = dudx[3 * in + d] * facn + dudx[3 * ip + d] * facp;
                dv[d] = dvdx[3 * in + d] * facn + dvdx[3 * ip + d] * facp;
                dw[d] = dwdx[3 * in + d] * facn + dwdx[3 * ip + d] * facp;
            }
            double visac = visC[in] * facn + visC[ip] * facp;
            sub3(m->cellCenter + 3 * in, m->cellCenter + 3 * ip, xpn);
            visFace = visac * rl;
            double mf = massFlux[i];
            double fuce = mf * uFace, fvce = mf * vFace, fwce = mf * wFace;
            double fude1 = (du[0] + du[0]) * S[0] + (du[1] + dv[0]) * S[1] + (du[2] + dw[0]) * S[2];
            double fvde1 = (du[1] + dv[0]) * S[0] + (dv[1] + dv[1]) * S[1] + (dv[2] + dw[1]) * S[2];
            double fwde1 = (du[2] + dw[0]) * S[0] + (dw[1] + dv[2]) * S[1] + (dw[2] + dw[2]) * S[2];
            double fude = visac * fude1, fvde = visac * fvde1, fwde = visac * fwde1;
            double fmin = std_min(mf, 0.0), fmax = std_max(mf, 0.0);
            double fuci = fmin * u[in] + fmax * u[ip];
            double fvci = fmin * v[in] + fmax * v[ip];
            double fwci = fmin * w[in] + fmax * w[ip];
            double fudi = visFace * dot3(du, xpn), fvdi = visFace * dot3(dv, xpn), fwdi = visFace * dot3(dw, xpn);
            rFace[2 * i] = -visFace - std_max(mf, 0.0);
            rFace[2 * i + 1] = -visFace + std_min(mf, 0.0);
            double bu = gammaBlend * (fuce - fuci), bv = gammaBlend * (fvce - fvci), bw = gammaBlend * (fwce - fwci);
            su[ip] = su[ip] - bu + fude - fudi;
            su[in] = su[in] + bu - fude + fudi;
            sv[ip] = sv[ip] - bv + fvde - fvdi;
            sv[in] = sv[in] + bv - fvde + fvdi;
            sw[ip] = sw[ip] - bw + fwde - fwdi;
            sw[in] = sw[in] + bw - fwde + fwdi;
            continue;
        }
        int ib = m->faceBnd[i], ir = m->bndRegion[ib], it = m->regionType[ir];
        const double *X = m->faceCenter + 3 * i;
        const double *du = dudx + 3 * ip, *dv = dvdx + 3 * ip, *dw = dwdx + 3 * ip;
        double xpn[3];
        sub3(X, m->cellCenter + 3 * ip, xpn);
        if (it == ORC_RTYPE_INLET || it == ORC_RTYPE_OUTLET) {
            double visac, fvde, fwde;
            double fude = (du[0] + du[0]) * S[0] + (du[1] + dv[0]) * S[1] + (du[2] + dw[0]) * S[2];
            if (it == ORC_RTYPE_INLET) {   /* UVWKernels.ipp:259-319 */
                uFace = m->regionUVW[3 * ir]; vFace = m->regionUVW[3 * ir + 1]; wFace = m->regionUVW[3 * ir + 2];
                visac = visB[ib];
                fvde = (du[1] + dv[0]) * S[0] + (dv[1] + dv[1]) * S[1] + (dv[2] + dw[1]) * S[2];
                fwde = (du[2] + dw[0]) * S[0] + (dw[1] + dv[2]) * S[1] + (dw[2] + dw[2]) * S[2];
            } else {                       /* UVWKernels.ipp:320-382 */
                visac = visC[ip];
                uFace = u[ip]; vFace = v[ip]; wFace = w[ip];
                fvde = (dv[0] + du[1]) * S[0] + (dv[1] + dv[1]) * S[1] + (dv[2] + dw[1]) * S[2];
                fwde = (dw[0] + du[2]) * S[0] + (dw[1] + dv[2]) * S[1] + (dw[2] + dw[2]) * S[2];
            }
            visFace = visac * rl;
            fude = visac * fude; fvde = visac * fvde; fwde = visac * fwde;
            double fudi = visFace * dot3(du, xpn), fvdi = visFace * dot3(dv, xpn), fwdi = visFace * dot3(dw, xpn);
            if (it == ORC_RTYPE_OUTLET && massFlux[i] < 0.0) massFlux[i] = small;
            double f = -visFace + std_min(massFlux[i], 0.0);
            au[ip] = au[ip] - f;
            su[ip] = su[ip] - f * uFace + fude - fudi;
            uB[ib] = uFace;
            av[ip] = av[ip] - f;
            sv[ip] = sv[ip] - f * vFace + fvde - fvdi;
            vB[ib] = vFace;
            aw[ip] = aw[ip] - f;
            sw[ip] = sw[ip] - f * wFace + fwde - fwdi;
            wB[ib] = wFace;
        } else if (it == ORC_RTYPE_SYMP) { /* UVWKernels.ipp:383-436; visFace carried, :424 */
            double visac = visC[ip];
            double us[3] = {u[ip] + dot3(du, xpn), v[ip] + dot3(dv, xpn), w[ip] + dot3(dw, xpn)};
            double xn[3] = {0.0 - S[0], 0.0 - S[1], 0.0 - S[2]};
            normalise3(xn);
            double dp = dot3(us, xn);
            double dn = bndDist ? bndDist[ib] : 0.0;
            double force[3];
            for (int d = 0; d < 3; d++) force[d] = (2.0 * visac * (dp * xn[d]) / dn) * m->faceArea[i];
            au[ip] = au[ip] + visFace;
            av[ip] = av[ip] + visFace;
            aw[ip] = aw[ip] + visFace;
            su[ip] = su[ip] + visFace * u[ip] - force[0];
            sv[ip] = sv[ip] + visFace * v[ip] - force[1];
            sw[ip] = sw[ip] + visFace * w[ip] - force[2];
            uB[ib] = us[0]; vB[ib] = us[1]; wB[ib] = us[2];
        } else if (it == ORC_RTYPE_WALL) { /* UVWKernels.ipp:437-510 */
            const double *uw = m->regionUVW + 3 * ir;
            double visac = visB[ib];
            double coef = visac * m->faceArea[i] / sqrt(dot3(xpn, xpn));
            double xn[3] = {S[0], S[1], S[2]};
            normalise3(xn);
            double up[3] = {u[ip] - uw[0], v[ip] - uw[1], w[ip] - uw[2]};
            double dp = dot3(up, xn);
            double ut[3] = {up[0] - dp * xn[0], up[1] - dp * xn[1], up[2] - dp * xn[2]};
            double uvel = fabs(ut[0]) + fabs(ut[1]) + fabs(ut[2]);
            double force[3] = {0.0, 0.0, 0.0};
            if (uvel > small) {
                double dn = bndDist ? bndDist[ib] : 0.0;
                for (int d = 0; d < 3; d++) force[d] = (visac * ut[d] / dn) * m->faceArea[i];
            }
            for (int d = 0; d < 3; d++) shear[3 * ib + d] = force[d];
            au[ip] = au[ip] + coef;
            av[ip] = av[ip] + coef;
            aw[ip] = aw[ip] + coef;
            su[ip] = su[ip] + coef * u[ip] - force[0];
            sv[ip] = sv[ip] + coef * v[ip] - force[1];
            sw[ip] = sw[ip] + coef * w[ip] - force[2];
            uB[ib] = uw[0]; vB[ib] = uw[1]; wB[ib] = uw[2];
        }
    }
    return ORC_E_SUCCESS;
}

/* FluxUVWDolfynRegionLoop1 (UVWKernels.ipp:517-524): every region's force
 * tangent set to zero. */
int orc_uvw_region_loop1(const orc_mesh *m, double *forceTangent) {
    for (int r = 0; r < 3 * m->nRegions; r++) forceTangent[r] = 0.0;
    return ORC_E_SUCCESS;
}

/* FluxUVWDolfynBndsLoop1 (UVWKernels.ipp:527-544): wall boundaries add their
 * shear onto their region's force tangent, in boundary order. */
int orc_uvw_bnds_loop1(const orc_mesh *m, const double *shear, double *forceTangent) {
    for (int ib = 0; ib < m->nBnd; ib++) {
        int ir = m->bndRegion[ib];
        if (m->regionType[ir] != ORC_RTYPE_WALL) continue;
        for (int d = 0; d < 3; d++) forceTangent[3 * ir + d] = forceTangent[3 * ir + d] + shear[3 * ib + d];
    }
    return ORC_E_SUCCESS;
}

/* ------------------------------------------------------------------------
 * The momentum loops of the reference's T = float instantiation
 * (UVWKernels.ipp:38-544 with T = float). Every product, sum and quotient
 * rounds in float in the reference's operand order, with three exceptions
 * the float build has:
 *   - facp = 1.0 - facn: the literal is double, the result rounded to float;
 *   - the wall branch's uvel = fabs(ut0) + fabs(ut1) + fabs(ut2): fabs is
 *     the C library's double function in the reference's scope, so the sum
 *     is double and rounds to float once on assignment (checked against the
 *     compiled float build in tests/test_oracle_vs_reference.py);
 *   - EuclideanVector::length() widens sqrtf's result to double, which the
 *     float scalars of normalise() and of the wall's xpn_length take back
 *     exactly (EuclideanVector.cpp:93-109), so both are the float sqrt.
 * 2.0 * visac (symmetry) is exact in double and exact again as float.
 * ------------------------------------------------------------------------ */
static float dot3f(const float *a, const float *b) {
    float d = 0.0f;
    for (int k = 0; k < 3; k++) d += a[k] * b[k];
    return d;
}
static void normalise3f(float *x) {
    float len = sqrtf(dot3f(x, x));
    if (len != 0.0f) {
        float sc = 1.0f / len;
        x[0] *= sc; x[1] *= sc; x[2] *= sc;
    }
}
static float std_minf(float a, float b) { return (b < a) ? b : a; }
static float std_maxf(float a, float b) { return (a < b) ? b : a; }

int orc_uvw_face_loop1_f32(const orc_mesh_f *m, const float *rlencos, const float *bndDist, float gammaBlend, float small,
                           const float *u, const float *v, const float *w, float *uB, float *vB, float *wB,
                           const float *visC, const float *visB, float *massFlux,
                           const float *dudx, const float *dvdx, const float *dwdx, float *rFace,
                           float *su, float *sv, float *sw, float *au, float *av, float *aw, float *shear) {
    float uFace = 0.0f, vFace = 0.0f, wFace = 0.0f, visFace = 0.0f;
    for (int i = 0; i < m->nFaces; i++) {
        int ip = m->faceCell1[i];
        const float *S = m->faceNorm + 3 * i;
        float rl = rlencos ? rlencos[i] : 0.0f;
        if (m->faceBnd[i] < 0) {
            int in = m->faceCell2[i];
            float facn = m->faceLambda[i];
            float facp = (float) (1.0 - (double) facn);
            float du[3], dv[3], dw[3], xpn[3];
            for (int d = 0; d < 3; d++) {
                du[d] = dudx[3 * in + d] * facn + dudx[3 * ip + d] * facp;
                dv[d] = dvdx[3 * in + d] * facn + dvdx[3 * ip + d] * facp;
                dw[d] = dwdx[3 * in + d] * facn + dwdx[3 * ip + d] * facp;
                xpn[d] = m->cellCenter[3 * in + d] - m->cellCenter[3 * ip + d];
            }
            float visac = visC[in] * facn + visC[ip] * facp;
            visFace = visac * rl;
            float mf = massFlux[i];
            float fuce = mf * uFace, fvce = mf * vFace, fwce = mf * wFace;
            float fude1 = (du[0] + du[0]) * S[0] + (du[1] + dv[0]) * S[1] + (du[2] + dw[0]) * S[2];
            float fvde1 = (du[1] + dv[0]) * S[0] + (dv[1] + dv[1]) * S[1] + (dv[2] + dw[1]) * S[2];
            float fwde1 = (du[2] + dw[0]) * S[0] + (dw[1] + dv[2]) * S[1] + (dw[2] + dw[2]) * S[2];
            float fude = visac * fude1, fvde = visac * fvde1, fwde = visac * fwde1;
            float fmin = std_minf(mf, 0.0f), fmax = std_maxf(mf, 0.0f);
            float fuci = fmin * u[in] + fmax * u[ip];
            float fvci = fmin * v[in] + fmax * v[ip];
            float fwci = fmin * w[in] + fmax * w[ip];
            float fudi = visFace * dot3f(du, xpn), fvdi = visFace * dot3f(dv, xpn), fwdi = visFace * dot3f(dw, xpn);
            rFace[2 * i] = -visFace - std_maxf(mf, 0.0f);
            rFace[2 * i + 1] = -visFace + std_minf(mf, 0.0f);
            float bu = gammaBlend * (fuce - fuci), bv = gammaBlend * (fvce - fvci), bw = gammaBlend * (fwce - fwci);
            su[ip] = su[ip] - bu + fude - fudi;
            su[in] = su[in] + bu - fude + fudi;
            sv[ip] = sv[ip] - bv + fvde - fvdi;
            sv[in] = sv[in] + bv - fvde + fvdi;
            sw[ip] = sw[ip] - bw + fwde - fwdi;
            sw[in] = sw[in] + bw - fwde + fwdi;
            continue;
        }
        int ib = m->faceBnd[i], ir = m->bndRegion[ib], it = m->regionType[ir];
        const float *X = m->faceCenter + 3 * i;
        const float *du = dudx + 3 * ip, *dv = dvdx + 3 * ip, *dw = dwdx + 3 * ip;
        float xpn[3];
        for (int d = 0; d < 3; d++) xpn[d] = X[d] - m->cellCenter[3 * ip + d];
        if (it == ORC_RTYPE_INLET || it == ORC_RTYPE_OUTLET) {
            float visac, fvde, fwde;
            float fude = (du[0] + du[0]) * S[0] + (du[1] + dv[0]) * S[1] + (du[2] + dw[0]) * S[2];
            if (it == ORC_RTYPE_INLET) {
                uFace = m->regionUVW[3 * ir]; vFace = m->regionUVW[3 * ir + 1]; wFace = m->regionUVW[3 * ir + 2];
                visac = visB[ib];
                fvde = (du[1] + dv[0]) * S[0] + (dv[1] + dv[1]) * S[1] + (dv[2] + dw[1]) * S[2];
                fwde = (du[2] + dw[0]) * S[0] + (dw[1] + dv[2]) * S[1] + (dw[2] + dw[2]) * S[2];
            } else {
                visac = visC[ip];
                uFace = u[ip]; vFace = v[ip]; wFace = w[ip];
                fvde = (dv[0] + du[1]) * S[0] + (dv[1] + dv[1]) * S[1] + (dv[2] + dw[1]) * S[2];
                fwde = (dw[0] + du[2]) * S[0] + (dw[1] + dv[2]) * S[1] + (dw[2] + dw[2]) * S[2];
            }
            visFace = visac * rl;
            fude = visac * fude; fvde = visac * fvde; fwde = visac * fwde;
            float fudi = visFace * dot3f(du, xpn), fvdi = visFace * dot3f(dv, xpn), fwdi = visFace * dot3f(dw, xpn);
            if (it == ORC_RTYPE_OUTLET && massFlux[i] < 0.0) massFlux[i] = small;
            float f = -visFace + std_minf(massFlux[i], 0.0f);
            au[ip] = au[ip] - f;
            su[ip] = su[ip] - f * uFace + fude - fudi;
            uB[ib] = uFace;
            av[ip] = av[ip] - f;
            sv[ip] = sv[ip] - f * vFace + fvde - fvdi;
            vB[ib] = vFace;
            aw[ip] = aw[ip] - f;
            sw[ip] = sw[ip] - f * wFace + fwde - fwdi;
            wB[ib] = wFace;
        } else if (it == ORC_RTYPE_SYMP) {
            float visac = visC[ip];
            float us[3] = {u[ip] + dot3f(du, xpn), v[ip] + dot3f(dv, xpn), w[ip] + dot3f(dw, xpn)};
            float xn[3] = {0.0f - S[0], 0.0f - S[1], 0.0f - S[2]};
            normalise3f(xn);
            float dp = dot3f(us, xn);
            float dn = bndDist ? bndDist[ib] : 0.0f;
            float tv = (float) (2.0 * (double) visac);
            float force[3];
            for (int d = 0; d < 3; d++) force[d] = ((tv * (dp * xn[d])) / dn) * m->faceArea[i];
            au[ip] = au[ip] + visFace;
            av[ip] = av[ip] + visFace;
            aw[ip] = aw[ip] + visFace;
            su[ip] = su[ip] + visFace * u[ip] - force[0];
            sv[ip] = sv[ip] + visFace * v[ip] - force[1];
            sw[ip] = sw[ip] + visFace * w[ip] - force[2];
            uB[ib] = us[0]; vB[ib] = us[1]; wB[ib] = us[2];
        } else if (it == ORC_RTYPE_WALL) {
            const float *uw = m->regionUVW + 3 * ir;
            float visac = visB[ib];
            float coef = visac * m->faceArea[i] / sqrtf(dot3f(xpn, xpn));
            float xn[3] = {S[0], S[1], S[2]};
            normalise3f(xn);
            float up[3] = {u[ip] - uw[0], v[ip] - uw[1], w[ip] - uw[2]};
            float dp = dot3f(up, xn);
            float ut[3] = {up[0] - dp * xn[0], up[1] - dp * xn[1], up[2] - dp * xn[2]};
            float uvel = (float) (fabs((double) ut[0]) + fabs((double) ut[1]) + fabs((double) ut[2]));
            float force[3] = {0.0f, 0.0f, 0.0f};
            if (uvel > small) {
                float dn = bndDist ? bndDist[ib] : 0.0f;
                for (int d = 0; d < 3; d++) force[d] = ((visac * ut[d]) / dn) * m->faceArea[i];
            }
            for (int d = 0; d < 3; d++) shear[3 * ib + d] = force[d];
            au[ip] = au[ip] + coef;
            av[ip] = av[ip] + coef;
            aw[ip] = aw[ip] + coef;
            su[ip] = su[ip] + coef * u[ip] - force[0];
            sv[ip] = sv[ip] + coef * v[ip] - force[1];
            sw[ip] = sw[ip] + coef * w[ip] - force[2];
            uB[ib] = uw[0]; vB[ib] = uw[1]; wB[ib] = uw[2];
        }
    }
    return ORC_E_SUCCESS;
}

int orc_uvw_bnds_loop1_f32(const orc_mesh_f *m, const float *shear, float *forceTangent) {
    for (int ib = 0; ib < m->nBnd; ib++) {
        int ir = m->bndRegion[ib];
        if (m->regionType[ir] != ORC_RTYPE_WALL) continue;
        for (int d = 0; d < 3; d++) forceTangent[3 * ir + d] = forceTangent[3 * ir + d] + shear[3 * ib + d];
    }
    return ORC_E_SUCCESS;
}
