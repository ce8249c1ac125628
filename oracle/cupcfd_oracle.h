/*
 * cupcfd_oracle.h - plain-C restatement of the reference's CPU algorithm for
 * the finite-volume face-loop path (Gauss-Green gradient + face mass flux),
 * plus the structured mesh generator and the cell->face CSR build it runs on.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker for the CUDA library, never
 * the thing measured or shipped: only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it. The CUDA library does not link it.
 *
 * Pinned against: the reference's own golden vectors in
 * tests/geometry/mesh/implementation/source/MeshStructGenSourceTests.cpp
 * (fixtures in tests/golden/), and against the reference's own kernels and
 * generator compiled unchanged into oracle/_ref/libcupcfd_ref.so.
 *
 * Conventions: all arrays are flat; 3-vectors are xyz-interleaved [3*n];
 * indices are 0-based int32; FP64 throughout. Return values are the
 * reference's eCodes integers (include/error/Error.h:32-144).
 */
#ifndef CUPCFD_ORACLE_H
#define CUPCFD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* eCodes values of the reference enum (include/error/Error.h:32-144). */
#define ORC_E_ARRAY_SIZE_MISMATCH 25
#define ORC_E_INVALID_INDEX 68
#define ORC_E_SUCCESS 95
#define ORC_E_ERROR 98

/* RType (include/geometry/mesh/interface/component/UnstructuredMeshInterface.h:58-65) */
#define ORC_RTYPE_DEFAULT 0
#define ORC_RTYPE_INLET 1
#define ORC_RTYPE_OUTLET 2
#define ORC_RTYPE_SYMP 3
#define ORC_RTYPE_WALL 4

/* A one-rank CupCfdSoAMesh as the kernels see it
 * (src/geometry/mesh/implementation/component/CupCfdSoAMesh.cpp, CupCfdSoAMesh.ipp:41-271). */
typedef struct {
    int nCells, nFaces, nBnd, nRegions;
    const int *faceCell1, *faceCell2, *faceBnd;   /* faceCell2 = -1 / faceBnd = -1 as in addFace */
    const double *faceLambda, *faceNorm, *faceCenter, *faceArea, *faceXpac, *faceXnac;
    const double *cellCenter, *cellVolume;
    const int *bndRegion, *regionType;
    const double *regionUVW, *regionDen;
} orc_mesh;

/* ---- structured hex generator (MeshStructGenSource.cpp) ---- */
void orc_structgen_counts(int nx, int ny, int nz, int *nCells, int *nFaces, int *nBnd, int *nVerts);
int orc_structgen_build(int nx, int ny, int nz,
                        double xmin, double xmax, double ymin, double ymax, double zmin, double zmax,
                        int *faceCell1, int *faceCell2, int *faceBnd,
                        double *faceLambda, double *faceNorm, double *faceCenter, double *faceArea,
                        double *cellCenter, double *cellVolume, int *faceVert, double *vertCoords);
int orc_structgen_cell_face_labels(int nx, int ny, int nz, int *xadj, int *adj);

/* ---- jittered + permuted hex mesh (own geometry definition, see .c) ---- */
int orc_jitter_build(int nx, int ny, int nz, double jitter, unsigned long long seed, int permute,
                     int *faceCell1, int *faceCell2, int *faceBnd,
                     double *faceLambda, double *faceNorm, double *faceCenter, double *faceArea,
                     double *cellCenter, double *cellVolume, int *cellPerm, int *facePerm);

/* ---- cell->face CSR (CupCfdSoAMesh::updateCellFaceMap, CupCfdSoAMesh.cpp:549-668) ---- */
int orc_cell_face_csr(int nCells, int nFaces, const int *faceCell1, const int *faceCell2, int *xadj, int *adj);

/* ---- kernels ---- */
/* The same mesh with float geometry and region values: the arrays a
 * CupCfdSoAMesh<int,float,int> holds (the reference's T = float
 * instantiation, BenchmarkKernels.cpp:1134-1138). */
typedef struct {
    int nCells, nFaces, nBnd, nRegions;
    const int *faceCell1, *faceCell2, *faceBnd;
    const float *faceLambda, *faceNorm, *faceCenter, *faceArea, *faceXpac, *faceXnac;
    const float *cellCenter, *cellVolume;
    const int *bndRegion, *regionType;
    const float *regionUVW, *regionDen;
} orc_mesh_f;

int orc_gradient_phi_gauss(const orc_mesh *m, int nGradient,
                           const double *phi, int nPhi, const double *phiB, int nPhiB,
                           double *dPhidx, int nDPhidx, double *dPhidxo, int nDPhidxo);

int orc_flux_mass_face_loop(const orc_mesh *m,
                            const double *dudx, const double *dvdx, const double *dwdx, const double *dpdx,
                            const double *den, double *denB, const double *u, const double *v, const double *w,
                            double *massFlux, const double *p, const double *ar, double *su, double *rface,
                            double small, int *icinl, int *icout, int *icsym, int *icwal,
                            int solveTurbEnergy, int solveTurbDiss, int solveVisc, int solveEnthalpy,
                            const double *teC, double *teB, const double *edC, double *edB,
                            const double *visC, double *visB, const double *tC, double *tB);

/* Adjoints (new; no reference counterpart). Gradient with nGradient = 1:
 * given gbar[3*nCells] = dL/d(dPhidx), accumulate dL/dphi into phibar[nCells]
 * and dL/dphiB into phibBar[nBnd]. Plain mass flux m_f = rho_f (u_f . S_f):
 * given mbar[nFaces] = dL/dm_f (interior faces), accumulate into
 * rhobar/ubar/vbar/wbar[nCells]. Outputs are overwritten. */
int orc_gradient_adjoint(const orc_mesh *m, const double *gbar, double *phibar, double *phibBar);

/* ---- boundary / region loops (MassKernels.ipp:311-554) ----
 * getBoundaryFaceID is the inverse of faceBnd; splvl[nRegions] stands for
 * getRegionSplvl. Arguments follow the reference's order. */
int orc_boundary_loop1(const orc_mesh *m, const double *massFlux, double *flowin);
int orc_boundary_loop2(const orc_mesh *m, const double *massFlux, double *flowRegion, double *flowout);
int orc_boundary_loop3(const orc_mesh *m, double flowin, double *ratearea);
int orc_boundary_loop4(const orc_mesh *m, const double *splvl, double *massFlux, double *uB, double *vB, double *wB,
                       const double *denB, double ratearea, double *flowout);
int orc_boundary_loop5(const orc_mesh *m, double *massFlux, double *su, double *uB, double *vB, double *wB, double fact,
                       int solveU, int solveV, int solveW, const double *flowFact, double *flowout2);
int orc_region_loop(const orc_mesh *m, const double *splvl, double *flowFact, const double *flowRegion, double flowIn);
/* ---- momentum face loop (UVWKernels.ipp:38-544) ----
 * rlencos[nFaces] / bndDist[nBnd] stand for getFaceRLencos /
 * getBoundaryDistance (NULL = all zero, as MeshSource-built meshes hold);
 * shear[3*nBnd] receives setBoundaryShear; forceTangent[3*nRegions] stands
 * for the region force tangents. The carried face values the reference
 * leaves uninitialised start at 0. */
int orc_uvw_face_loop1(const orc_mesh *m, const double *rlencos, const double *bndDist, double gammaBlend, double small,
                       const double *u, const double *v, const double *w, double *uB, double *vB, double *wB,
                       const double *visC, const double *visB, double *massFlux,
                       const double *dudx, const double *dvdx, const double *dwdx, double *rFace,
                       double *su, double *sv, double *sw, double *au, double *av, double *aw, double *shear);
int orc_uvw_region_loop1(const orc_mesh *m, double *forceTangent);
int orc_uvw_bnds_loop1(const orc_mesh *m, const double *shear, double *forceTangent);
/* The momentum loops of the reference's T = float instantiation: the same
 * loops with float arrays and the float build's arithmetic (see .c). */
int orc_uvw_face_loop1_f32(const orc_mesh_f *m, const float *rlencos, const float *bndDist, float gammaBlend, float small,
                           const float *u, const float *v, const float *w, float *uB, float *vB, float *wB,
                           const float *visC, const float *visB, float *massFlux,
                           const float *dudx, const float *dvdx, const float *dwdx, float *rFace,
                           float *su, float *sv, float *sw, float *au, float *av, float *aw, float *shear);
int orc_uvw_bnds_loop1_f32(const orc_mesh_f *m, const float *shear, float *forceTangent);
int orc_mass_plain_forward(const orc_mesh *m, const double *den, const double *u, const double *v, const double *w,
                           double *massFlux);
int orc_mass_plain_adjoint(const orc_mesh *m, const double *den, const double *u, const double *v, const double *w,
                           const double *mbar, double *denbar, double *ubar, double *vbar, double *wbar);

#ifdef __cplusplus
}
#endif
#endif
