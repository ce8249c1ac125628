/*
 * cupcfd_gpu.h - C ABI of the B200 (sm_100a) implementation of CUP-CFD's
 * finite-volume face-loop path: the Gauss-Green cell gradient
 * (GradientPhiGaussDolfyn) and the face mass-flux loop
 * (FluxMassDolfynFaceLoop) over the reference's MiniSoA mesh, with their
 * adjoints; and the operators either side of it: the mass boundary / region
 * loops (FluxMassDolfynBoundaryLoop1-5, FluxMassDolfynRegionLoop), the
 * momentum face loop (FluxUVWDolfynFaceLoop1, RegionLoop1, BndsLoop1) and
 * mesh files.
 *
 * Plain C: pointers, sizes and int status codes only. Status codes are the
 * reference's eCodes values (include/error/Error.h:32-144): CUPCFD_E_SUCCESS
 * is E_SUCCESS, and so on. No call aborts; CUDA failures map to
 * CUPCFD_E_ERROR and the message is available from cupcfd_gpu_last_error().
 *
 * Two layers:
 *  1. Reference-facing calls (cupcfd_gpu_gradient_phi_gauss_dolfyn,
 *     cupcfd_gpu_flux_mass_dolfyn_*, cupcfd_gpu_flux_uvw_dolfyn_*): HOST buffers in the
 *     reference's numbering and layout, including the 32-byte (double) /
 *     24-byte (float) stride of the vptr-carrying EuclideanVector<T,3>
 *     arrays. Each call copies inputs to the device, runs, and copies the
 *     outputs back before returning, exactly like the synchronous CPU call
 *     it replaces.
 *  2. Device-resident calls (cupcfd_gpu_dev_*): DEVICE pointers in the
 *     mesh's internal (renumbered) order, stream-ordered on the stream the
 *     caller passes, no host synchronisation. Fields are moved between the
 *     two numberings with cupcfd_gpu_dev_permute_cells / _permute_faces.
 *
 * Threading: a mesh handle is not thread-safe (as the reference mesh is
 * not); calls on one handle must be serialised by the caller.
 */
#ifndef CUPCFD_GPU_H
#define CUPCFD_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: values of the reference enum cupcfd::error::eCodes ---- */
#define CUPCFD_E_ARRAY_SIZE_MISMATCH 25 /* E_ARRAY_SIZE_MISMATCH, Error.h:59 */
#define CUPCFD_E_INVALID_INDEX 68       /* E_INVALID_INDEX, Error.h:102 */
#define CUPCFD_E_CONFIG_INVALID_VALUE 90 /* E_CONFIG_INVALID_VALUE, Error.h:124 */
#define CUPCFD_E_SUCCESS 95             /* E_SUCCESS, Error.h:129 */
#define CUPCFD_E_ERROR 98               /* E_ERROR, Error.h:132 */
#define CUPCFD_E_NULL_PTR 99            /* E_NULL_PTR, Error.h:133 */
#define CUPCFD_E_NOT_IMPLEMENTED 109    /* E_NOT_IMPLEMENTED, Error.h:143 */
#define CUPCFD_E_FILE_MISSING 10        /* E_FILE_MISSING, Error.h:44 */
#define CUPCFD_E_INVALID_FILE_FORMAT 105 /* E_INVALID_FILE_FORMAT, Error.h:139 */
#define CUPCFD_E_CONFIG_OPT_NOT_FOUND 92 /* E_CONFIG_OPT_NOT_FOUND, Error.h:126 */

/* ---- region types: cupcfd::geometry::mesh::RType (UnstructuredMeshInterface.h:58-65) ---- */
#define CUPCFD_RTYPE_DEFAULT 0
#define CUPCFD_RTYPE_INLET 1
#define CUPCFD_RTYPE_OUTLET 2
#define CUPCFD_RTYPE_SYMP 3
#define CUPCFD_RTYPE_WALL 4

/* ---- arithmetic of a call ---- */
#define CUPCFD_PREC_F64 0  /* plain FP64; same operand order as the reference, bit-identical results */
#define CUPCFD_PREC_F32C 1 /* FP32 storage and arithmetic, compensated (TwoSum) cell accumulation,
                              FP64 volumes and final scaling */
#define CUPCFD_PREC_F32REF 2 /* gradient calls only: the arithmetic of the reference's T=float
                                instantiation (float sums in its order), bit-identical to it on a
                                mesh uploaded from the same float arrays; uses the FP32 geometry */

/* ---- internal numbering of a device mesh ---- */
#define CUPCFD_ORDER_NATIVE 0 /* cells and faces in the reference's local order */
#define CUPCFD_ORDER_MORTON 1 /* cells by Z-order of their centres, faces by owner (see below) */
#define CUPCFD_ORDER_OWNER 2  /* cells in reference order, faces by owner (see below) */
#define CUPCFD_ORDER_RCM 3    /* cells by reverse Cuthill-McKee, faces by owner (see below) */
/* "Faces by owner": sorted by (owner's 32-cell slice, rank of the face among
 * its owner's faces, owner's lane in the slice), so that the k-th face of 32
 * consecutive cells are consecutive records. */

/* ---- gradient sign convention ---- */
#define CUPCFD_SIGN_REFERENCE 0 /* phi_f S_f added to BOTH cells with the same sign,
                                   as GradientKernels.ipp:102-103 does (default) */
#define CUPCFD_SIGN_SIGNED 1    /* textbook Gauss-Green: the neighbour subtracts */

/* Strided view of an array of 3-vectors: component d (0..2) of element i is
 * the real at (char*)base + i*stride + offset + d*real_size. For a
 * std::vector<EuclideanVector<double,3>> stride = 32 and offset = 8 (the
 * vptr); for a packed xyz array stride = 3*real_size and offset = 0. */
typedef struct {
    const void *base;
    int32_t stride;
    int32_t offset;
} cupcfd_vec3_view;

/* Host view of a one-rank CupCfdSoAMesh<int,T,int> (CupCfdSoAMesh.h:59-558):
 * the arrays its getters read, indexed by local id. real_size is sizeof(T)
 * (8 or 4) and applies to every real array and vector view. faceCell2 is -1
 * and faceBnd is the local boundary id on boundary faces; faceBnd is -1 on
 * interior faces (CupCfdSoAMesh.cpp:309-461). faceXpac/faceXnac may have a
 * NULL base, meaning all zero (what addData stores, UnstructuredMeshInterface.ipp:1778-1780). */
typedef struct {
    int32_t nCells;      /* properties.lTCells */
    int32_t nFaces;      /* properties.lFaces */
    int32_t nBoundaries; /* properties.lBoundaries */
    int32_t real_size;   /* 8 (double) or 4 (float) */
    const int32_t *faceCell1;
    const int32_t *faceCell2;
    const int32_t *faceBnd;
    const void *faceLambda;
    const void *faceArea;
    cupcfd_vec3_view faceNorm;
    cupcfd_vec3_view faceCenter;
    cupcfd_vec3_view faceXpac;
    cupcfd_vec3_view faceXnac;
    cupcfd_vec3_view cellCenter;
    const void *cellVolume;
} cupcfd_mesh_view;

typedef struct {
    int32_t order;      /* CUPCFD_ORDER_* */
    int32_t precisions; /* bit mask: 1 << CUPCFD_PREC_F64 | 1 << CUPCFD_PREC_F32C */
    int32_t device;     /* CUDA device ordinal, -1 = current */
} cupcfd_mesh_options;

typedef struct {
    int32_t nCells, nFaces, nInteriorFaces, nBoundaries, nRegions;
    int32_t nIncidences; /* 2*interior + boundary faces: length of the cell->face CSR */
    int32_t maxCellFaces;
    int32_t order, precisions;
    int32_t bandwidth;   /* largest |c - neighbour| of the internal numbering */
    int64_t deviceBytes; /* device memory held by the mesh */
    int32_t tiles;       /* 1 when the face loops take the L2-prefetch kernels (faces numbered by owner tile) */
    int32_t fullWidth;   /* 6 when those kernels run their six-incidence specialisation (every cell has six
                            faces: hexahedral meshes), else 0 */
} cupcfd_mesh_info;

typedef struct cupcfd_gpu_mesh cupcfd_gpu_mesh;

/* Message of the last failing call on this thread ("" if none). */
const char *cupcfd_gpu_last_error(void);
/* Library version string. */
const char *cupcfd_gpu_version(void);

/* ------------------------------------------------------------------------ */
/* mesh                                                                      */
/* ------------------------------------------------------------------------ */

/* Uploads a host mesh, validates its connectivity, builds the cell->face CSR
 * exactly as CupCfdSoAMesh::updateCellFaceMap does (CupCfdSoAMesh.cpp:549-668),
 * renumbers, and lays out the device arrays. One region of type
 * RTYPE_DEFAULT is installed; see cupcfd_gpu_mesh_set_regions.
 * Replaces: the CupCfdSoAMesh finalize()/addData() result the reference
 * kernels read (CupCfdSoAMesh.cpp:842-888). */
int cupcfd_gpu_mesh_create(const cupcfd_mesh_view *view, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out);

/* Builds the structured hex mesh of MeshStructGenSource(nx, ny, nz, bounds)
 * (src/geometry/mesh/implementation/source/MeshStructGenSource.cpp:33-1277)
 * directly on the GPU in FP64, in the reference's label order, then proceeds
 * as cupcfd_gpu_mesh_create. bounds = {xmin, xmax, ymin, ymax, zmin, zmax}.
 * Cell volumes are the box volume; the reference's five-tetrahedron Heron
 * sum agrees to 2e-14 relative (its own rounding). */
int cupcfd_gpu_mesh_create_structgen(int32_t nx, int32_t ny, int32_t nz, const double bounds[6],
                                     const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out);

/* Unit-cube hex mesh with every interior vertex displaced by
 * U[-jitter*h, jitter*h] per axis (splitmix64 stream keyed by seed, vertex,
 * axis) and, if permute != 0, cell and face labels shuffled by seeded
 * Fisher-Yates permutations. Geometry: S_f = 0.5 (v2-v0) x (v3-v1) oriented
 * away from cell1, area |S_f|, face centre = vertex mean, cell centre =
 * vertex mean, volume = sum_f x_f . S_f,out / 3, lambda = ((x_f - x_1) . S) /
 * ((x_2 - x_1) . S). Used for the irregular-mesh workload; no reference
 * counterpart (the reference reads such meshes from HDF5, MeshHDF5Source.cpp). */
int cupcfd_gpu_mesh_create_jittered(int32_t nx, int32_t ny, int32_t nz, double jitter, uint64_t seed, int32_t permute,
                                    const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out);

/* Mesh files of this library (the reference's own HDF5 mesh files are read
 * and written by the cupcfd_gpu_hdf5_* calls below). A device mesh is saved
 * to, and reloaded from, a raw-binary file holding everything the device
 * mesh holds, its source arrays in the reference's numbering:
 * a 64-byte header (magic "CUPCFDM1", version 2, nCells, nFaces,
 * nBoundaries, nRegions, flags: bit 0 xpac/xnac present, bit 1 rlencos
 * present, bit 2 boundary distances present), then faceCell1, faceCell2,
 * faceBnd (int32), faceLambda, faceArea, faceNorm[3], faceCenter[3],
 * [faceXpac[3], faceXnac[3]], cellCenter[3], cellVolume (float64),
 * regionType (int32), regionUVW[3], regionDen, regionSplvl (float64),
 * bndRegion (int32), [faceRLencos], [boundaryDistance] (float64), and an
 * FNV-1a 64-bit checksum of all the bytes before it, taken over 64-bit
 * little-endian words (h = (h ^ word) * 1099511628211 from
 * 14695981039346656037; a last partial word padded with zero bytes).
 * Little-endian. Loading rebuilds the device layout exactly as
 * cupcfd_gpu_mesh_create with `opt`, then installs the regions, split
 * levels, rlencos and boundary distances, so kernels on a loaded mesh give
 * the saved mesh's bits.
 * Errors: CUPCFD_E_FILE_MISSING (cannot open), CUPCFD_E_INVALID_FILE_FORMAT
 * (magic, version, header ranges, size, truncation or hash wrong), as the
 * reference's readers return (Error.h:44, Error.h:139). */
int cupcfd_gpu_mesh_save(const cupcfd_gpu_mesh *mesh, const char *path);
int cupcfd_gpu_mesh_load(const char *path, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out);

/* Mesh ingest from the reference's HDF5 mesh files, as MeshHDF5Source reads
 * them (src/geometry/mesh/implementation/source/MeshHDF5Source.cpp:42-1130)
 * and addData lays them out on one rank (UnstructuredMeshInterface.ipp:
 * 1464-1862): root attributes ncel, nfac, nbnd, nreg; /face/{cell1, cell2,
 * bnd, lambda, area, n, x}, /cell/{x, vol}, /bnd/{rid, distance}; 1-based
 * labels; cell2 = 0 marks a boundary face. The library reads the HDF5 format
 * itself (superblock 0/1, symbol-table groups, version-1 object headers,
 * compact or contiguous little-endian datasets; an unallocated dataset reads
 * as its fill value); other files return CUPCFD_E_INVALID_FILE_FORMAT, a
 * missing one CUPCFD_E_FILE_MISSING, labels out of range CUPCFD_E_INVALID_INDEX.
 *   counts: the four root attributes;
 *   read:   the arrays in the reference's (0-based) numbering into host
 *           buffers (any may be NULL): faceCell1/2, faceBnd [nFaces] (-1 on
 *           interior faces / cell2 of boundary faces), faceLambda, faceArea
 *           [nFaces], faceNorm, faceCenter [3*nFaces], cellCenter [3*nCells],
 *           cellVolume [nCells], bndRegion, bndDistance [nBoundaries];
 *   load:   the device mesh, with default regions, the boundaries' regions
 *           and distances. */
int cupcfd_gpu_hdf5_mesh_counts(const char *path, int32_t *nCells, int32_t *nFaces, int32_t *nBoundaries,
                                int32_t *nRegions);
int cupcfd_gpu_hdf5_mesh_read(const char *path, int32_t nCells, int32_t nFaces, int32_t nBoundaries, int32_t *faceCell1,
                              int32_t *faceCell2, int32_t *faceBnd, double *faceLambda, double *faceArea,
                              double *faceNorm, double *faceCenter, double *cellCenter, double *cellVolume,
                              int32_t *bndRegion, double *bndDistance);
int cupcfd_gpu_mesh_load_hdf5(const char *path, const cupcfd_mesh_options *opt, cupcfd_gpu_mesh **out);

/* Mesh files in the same HDF5 layout, written by the library (the datasets
 * MeshHDF5Source.cpp:215-1130 reads for connectivity and geometry): root
 * attributes ncel, nfac, nbnd, nreg and nvrt (0: no vertices are stored, so
 * /vert, /face/vertices and /bnd/vertices are absent); /cell/{nfaces, cface
 * ([nCells][max faces], each cell's face labels ascending, 0-padded), x, vol};
 * /face/{cell1, cell2 (0 on boundary faces), bnd (0 on interior faces),
 * lambda, area, n, x}; /bnd/{face, rid, distance}; labels 1-based.
 *   write:      host arrays as cupcfd_gpu_hdf5_mesh_read returns them
 *               (0-based; bndRegion and bndDistance may be NULL: region 0,
 *               distance 0). Face cells out of range, or boundary ids that
 *               are not one per boundary face, return CUPCFD_E_INVALID_INDEX;
 *               a file that cannot be created CUPCFD_E_FILE_MISSING;
 *   save:       a device mesh, its boundaries' regions and distances (region
 *               types are not part of the format: loading gives default
 *               regions, as for the reference's files);
 *   dataset:    any numeric dataset of such a file by path ("/cell/cface"):
 *               its shape (up to 4 dimensions, isReal 0 for integers), and
 *               its values as doubles (row-major, n = the element count). */
int cupcfd_gpu_hdf5_mesh_write(const char *path, int32_t nCells, int32_t nFaces, int32_t nBoundaries,
                               int32_t nRegions, const int32_t *faceCell1, const int32_t *faceCell2,
                               const int32_t *faceBnd, const double *faceLambda, const double *faceArea,
                               const double *faceNorm, const double *faceCenter, const double *cellCenter,
                               const double *cellVolume, const int32_t *bndRegion, const double *bndDistance);
int cupcfd_gpu_mesh_save_hdf5(const cupcfd_gpu_mesh *mesh, const char *path);
int cupcfd_gpu_hdf5_dataset_shape(const char *path, const char *name, int32_t *ndims, int64_t *dims,
                                  int32_t *isReal);
int cupcfd_gpu_hdf5_dataset_read(const char *path, const char *name, double *out, int64_t n);

int cupcfd_gpu_mesh_destroy(cupcfd_gpu_mesh *mesh);
int cupcfd_gpu_mesh_get_info(const cupcfd_gpu_mesh *mesh, cupcfd_mesh_info *info);

/* Synchronises `stream` (the asynchronous device calls' stream) and returns
 * CUPCFD_E_ERROR (message in cupcfd_gpu_last_error) if the work on it
 * failed, CUPCFD_E_SUCCESS otherwise. No kernel of this library waits on
 * another block, a peer or a flag, so a failed launch is the only
 * asynchronous error there is. */
int cupcfd_gpu_mesh_check_status(cupcfd_gpu_mesh *mesh, void *stream);

/* Boundary regions (CupCfdSoAMesh region/boundary arrays): regionType[nRegions]
 * (CUPCFD_RTYPE_*), regionUVW[3*nRegions], regionDen[nRegions] (host, real_size
 * 8) and bndRegion[nBoundaries] (host). Replaces getBoundaryRegionID /
 * getRegionType / getRegionUVW / getRegionDen (UnstructuredMeshInterface.h:1306-1949). */
int cupcfd_gpu_mesh_set_regions(cupcfd_gpu_mesh *mesh, int32_t nRegions, const int32_t *regionType,
                                const double *regionUVW, const double *regionDen,
                                const int32_t *bndRegion, int32_t nBoundaries);

/* Region split levels splvl[nRegions] (replaces getRegionSplvl,
 * UnstructuredMeshInterface.h:1855-1868), read by the outlet boundary loops;
 * zero until set, and reset to zero by cupcfd_gpu_mesh_set_regions. */
int cupcfd_gpu_mesh_set_region_split(cupcfd_gpu_mesh *mesh, int32_t nRegions, const double *splvl);

/* Downloads the cell->face CSR in the reference's numbering (host arrays,
 * xadj[nCells+1], adj[nIncidences]) for bit-exact comparison with
 * CupCfdSoAMesh::cellFaceMapCSRXAdj / cellFaceMapCSRAdj. */
int cupcfd_gpu_mesh_get_cell_face_csr(const cupcfd_gpu_mesh *mesh, int32_t *xadj, int32_t nXAdj, int32_t *adj, int32_t nAdj);

/* Downloads the incidence lists the face-loop kernels read, in the mesh's
 * internal numbering, as a CSR over internal cells (host arrays xadj[nCells+1],
 * face[nIncidences], other[nIncidences]): face = internal face id << 1 | role
 * (0 when the cell is the face's cell1, 1 when it is its cell2), other = the
 * face's other internal cell or -1 - boundaryId. Mapped back through
 * cupcfd_gpu_mesh_get_numbering, cell c's list equals row cellN2O[c] of
 * CupCfdSoAMesh::cellFaceMapCSRAdj, in order. No counterpart in the reference
 * (it checks a renumbering). */
int cupcfd_gpu_mesh_get_incidences(const cupcfd_gpu_mesh *mesh, int32_t *xadj, int32_t nXAdj, int32_t *face,
                                   int32_t *other, int32_t nInc);

/* Downloads the FP64 source arrays in the reference's numbering (any pointer
 * may be NULL): faceCell1/2, faceBnd [nFaces], faceLambda, faceArea [nFaces],
 * faceNorm, faceCenter [3*nFaces], cellCenter [3*nCells], cellVolume [nCells]. */
int cupcfd_gpu_mesh_get_geometry(const cupcfd_gpu_mesh *mesh, int32_t *faceCell1, int32_t *faceCell2, int32_t *faceBnd,
                                 double *faceLambda, double *faceArea, double *faceNorm, double *faceCenter,
                                 double *cellCenter, double *cellVolume);

/* Internal numbering: cellNew2Old[nCells], faceNew2Old[nFaces] (host, may be NULL). */
int cupcfd_gpu_mesh_get_numbering(const cupcfd_gpu_mesh *mesh, int32_t *cellNew2Old, int32_t *faceNew2Old);

/* ------------------------------------------------------------------------ */
/* reference-facing calls (host buffers, reference numbering and layout)     */
/* ------------------------------------------------------------------------ */

/* GradientPhiGaussDolfyn (include/fvm/implementation/component/GradientKernels.h:48-54,
 * GradientKernels.ipp:38-136). phiCell[nPhiCell], phiBoundary[nPhiBoundary]
 * are host arrays of real_size (4 or 8) bytes; dPhidxCell / dPhidxoCell are
 * host EuclideanVector<T,3> arrays seen through strided views (only the three
 * components are written; the vptr slot is never touched). nGradient
 * iterations with the non-orthogonal correction of the previous iterate.
 * precision: CUPCFD_PREC_F64 (bit-identical to the reference for T=double)
 * or CUPCFD_PREC_F32C; for T=float arrays (real_size 4) CUPCFD_PREC_F32REF
 * reproduces the reference's float instantiation bit for bit on a mesh
 * created from the same float arrays (PREC_F64 computes in FP64 and rounds
 * each result to float once; PREC_F32C is the compensated FP32 path).
 * sign_mode: CUPCFD_SIGN_*. */
int cupcfd_gpu_gradient_phi_gauss_dolfyn(cupcfd_gpu_mesh *mesh, int32_t nGradient,
                                         const void *phiCell, int32_t nPhiCell,
                                         const void *phiBoundary, int32_t nPhiBoundary,
                                         void *dPhidxCell, int32_t nDPhidxCell, int32_t stride, int32_t offset,
                                         void *dPhidxoCell, int32_t nDPhidxoCell, int32_t strideo, int32_t offseto,
                                         int32_t real_size, int32_t precision, int32_t sign_mode);

/* FluxMassDolfynFaceLoop (include/fvm/implementation/component/MassKernels.h:48-81,
 * MassKernels.ipp:36-309), full semantics: gradient-corrected face velocities,
 * the Rhie-Chow pressure term written to rface[2*nFaces], and the boundary
 * region branches (inlet: su[ip] -= flux; outlet: denBoundary and, for
 * backflow, te/ed/viseff/t boundary copies; symmetry/wall: zero flux),
 * updating the four counters. All arrays are host, FP64, reference layout;
 * dudx/dvdx/dwdx/dpdx are EuclideanVector<double,3> views. Arrays the
 * reference would not touch are not written. */
int cupcfd_gpu_flux_mass_dolfyn_face_loop(cupcfd_gpu_mesh *mesh,
                                          cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx,
                                          cupcfd_vec3_view dwdx, int32_t nDwdx, cupcfd_vec3_view dpdx, int32_t nDpdx,
                                          const double *denCell, int32_t nDenCell, double *denBoundary, int32_t nDenBoundary,
                                          const double *uCell, int32_t nUCell, const double *vCell, int32_t nVCell,
                                          const double *wCell, int32_t nWCell, double *massFlux, int32_t nMassFlux,
                                          const double *p, int32_t nP, const double *ar, int32_t nAr,
                                          double *su, int32_t nSu, double *rface, int32_t nRFace, double small,
                                          int32_t *icinl, int32_t *icout, int32_t *icsym, int32_t *icwal,
                                          int32_t solveTurbEnergy, int32_t solveTurbDiss, int32_t solveVisc, int32_t solveEnthalpy,
                                          const double *teCell, int32_t nTeCell, double *teBoundary, int32_t nTeBoundary,
                                          const double *edCell, int32_t nEdCell, double *edBoundary, int32_t nEdBoundary,
                                          const double *viseffCell, int32_t nViseffCell, double *viseffBoundary, int32_t nViseffBoundary,
                                          const double *tCell, int32_t nTCell, double *tBoundary, int32_t nTBoundary);

/* FluxMassDolfynFaceLoop of the reference's T = float instantiation
 * (BenchmarkKernels.cpp:1134-1138 instantiates the kernels for
 * CupCfdSoAMesh<int,float,int>): the same parameters with float arrays and
 * EuclideanVector<float,3> views (24-byte stride, components at +8), and the
 * float instantiation's own arithmetic (float products and sums in the
 * reference's order; 1.0 - lambda in double, rounded to float), on the
 * mesh's FP32 geometry, which a mesh uploaded from float arrays holds
 * exactly. Results are those of the reference's float build bit for bit.
 * The mesh must have CUPCFD_PREC_F32C geometry. */
int cupcfd_gpu_flux_mass_dolfyn_face_loop_f32(cupcfd_gpu_mesh *mesh,
                                              cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx,
                                              cupcfd_vec3_view dwdx, int32_t nDwdx, cupcfd_vec3_view dpdx, int32_t nDpdx,
                                              const float *denCell, int32_t nDenCell, float *denBoundary, int32_t nDenBoundary,
                                              const float *uCell, int32_t nUCell, const float *vCell, int32_t nVCell,
                                              const float *wCell, int32_t nWCell, float *massFlux, int32_t nMassFlux,
                                              const float *p, int32_t nP, const float *ar, int32_t nAr,
                                              float *su, int32_t nSu, float *rface, int32_t nRFace, float small,
                                              int32_t *icinl, int32_t *icout, int32_t *icsym, int32_t *icwal,
                                              int32_t solveTurbEnergy, int32_t solveTurbDiss, int32_t solveVisc, int32_t solveEnthalpy,
                                              const float *teCell, int32_t nTeCell, float *teBoundary, int32_t nTeBoundary,
                                              const float *edCell, int32_t nEdCell, float *edBoundary, int32_t nEdBoundary,
                                              const float *viseffCell, int32_t nViseffCell, float *viseffBoundary, int32_t nViseffBoundary,
                                              const float *tCell, int32_t nTCell, float *tBoundary, int32_t nTBoundary);

/* Forward + adjoint of the plain face loops through host buffers (the
 * benchmark's end-to-end call). Inputs (host, reference numbering, FP64):
 * phi[nCells], phiB[nBoundaries], den/u/v/w[nCells], gface[nFaces] (loss
 * weights). Loss L = sum_c V_c |dPhidx_c|^2 + sum_{interior f} gface_f m_f,
 * with m_f = rho_f (u_f . S_f). Outputs (host, FP64, any may be NULL):
 * grad[3*nCells] (xyz interleaved), massFlux[nFaces] (boundary entries 0),
 * phiBar[nCells], phiBBar[nBoundaries], denBar/uBar/vBar/wBar[nCells],
 * loss[1]. nGradient is 1. The inputs go in on a copy-in stream of the mesh
 * and the results come back on a copy-out stream while later inputs are
 * still being copied in (gradient and phiBar once phi is in, mass fluxes once
 * the state is in, the state adjoint and then the loss once gface is in);
 * they equal cupcfd_gpu_dev_forward_adjoint's bit for bit.
 * Pinned host buffers let the copies in both directions overlap. Returns when
 * every output is in host memory. */
int cupcfd_gpu_forward_adjoint(cupcfd_gpu_mesh *mesh, int32_t precision,
                               const double *phi, const double *phiB, const double *den, const double *u,
                               const double *v, const double *w, const double *gface,
                               double *grad, double *massFlux, double *phiBar, double *phiBBar,
                               double *denBar, double *uBar, double *vBar, double *wBar, double *loss);
/* The same call on float host arrays (the reference's T = float arrays):
 * half the bytes cross the host link. With CUPCFD_PREC_F32C the kernels see
 * exactly the values the FP64-array call gives them after its conversion,
 * so every output is that call's, rounded to float (exactly: the FP32 path's
 * outputs are float values). The loss stays double. */
int cupcfd_gpu_forward_adjoint_f32(cupcfd_gpu_mesh *mesh, int32_t precision,
                                   const float *phi, const float *phiB, const float *den, const float *u,
                                   const float *v, const float *w, const float *gface,
                                   float *grad, float *massFlux, float *phiBar, float *phiBBar,
                                   float *denBar, float *uBar, float *vBar, float *wBar, double *loss);

/* The boundary / region loops of the mass-flux step, FP64, bit-identical to
 * the reference (MassKernels.h:90-171, MassKernels.ipp:311-554): host
 * buffers in the reference's numbering (faces, cells, boundary ids, region
 * ids). Sums run in the reference's boundary order; array lengths below
 * the mesh's return E_INVALID_INDEX.
 *   loop1: flowin = sum of massFlux over inlet boundaries
 *   loop2: flowout = sum over outlets, flowRegion[region] += the same
 *   loop3: ratearea = -flowin / (outlet area)
 *   loop4: outlet massFlux = ratearea * area * splvl, outlet velocities
 *          along the unit normal, flowout = their sum
 *   loop5: outlet massFlux *= flowFact[region], *flowout2 += it (not reset),
 *          u/v/wBoundary *= fact where solveU/V/W, su[cell1] -= massFlux
 *   region loop: flowFact = -(splvl * flowIn) / flowRegion on outlets, else 0 */
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop1(cupcfd_gpu_mesh *mesh, const double *massFlux, int32_t nMassFlux,
                                               double *flowin);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop2(cupcfd_gpu_mesh *mesh, const double *massFlux, int32_t nMassFlux,
                                               double *flowRegion, int32_t nFlowRegion, double *flowout);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop3(cupcfd_gpu_mesh *mesh, double flowin, double *ratearea);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop4(cupcfd_gpu_mesh *mesh, double *massFlux, int32_t nMassFlux,
                                               double *uBoundary, int32_t nUBoundary, double *vBoundary,
                                               int32_t nVBoundary, double *wBoundary, int32_t nWBoundary,
                                               const double *denBoundary, int32_t nDenBoundary, double ratearea,
                                               double *flowout);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop5(cupcfd_gpu_mesh *mesh, double *massFlux, int32_t nMassFlux,
                                               double *su, int32_t nSu, double *uBoundary, int32_t nUBoundary,
                                               double *vBoundary, int32_t nVBoundary, double *wBoundary,
                                               int32_t nWBoundary, double fact, int32_t solveU, int32_t solveV,
                                               int32_t solveW, const double *flowFact, int32_t nFlowFact,
                                               double *flowout2);
int cupcfd_gpu_flux_mass_dolfyn_region_loop(cupcfd_gpu_mesh *mesh, double *flowFact, int32_t nFlowFact,
                                           const double *flowRegion, int32_t nFlowRegion, double flowIn);

/* The same loops, the reference's T = float instantiation
 * (MassKernels.ipp:311-554 with T = float): float host arrays, float
 * arithmetic in the reference's order, bit-identical to it. The mesh's
 * geometry and split levels enter rounded to float (exact for a mesh made
 * from float arrays, as the reference's float mesh is). */
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop1_f32(cupcfd_gpu_mesh *mesh, const float *massFlux, int32_t nMassFlux,
                                                   float *flowin);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop2_f32(cupcfd_gpu_mesh *mesh, const float *massFlux, int32_t nMassFlux,
                                                   float *flowRegion, int32_t nFlowRegion, float *flowout);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop3_f32(cupcfd_gpu_mesh *mesh, float flowin, float *ratearea);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop4_f32(cupcfd_gpu_mesh *mesh, float *massFlux, int32_t nMassFlux,
                                                   float *uBoundary, int32_t nUBoundary, float *vBoundary,
                                                   int32_t nVBoundary, float *wBoundary, int32_t nWBoundary,
                                                   const float *denBoundary, int32_t nDenBoundary, float ratearea,
                                                   float *flowout);
int cupcfd_gpu_flux_mass_dolfyn_boundary_loop5_f32(cupcfd_gpu_mesh *mesh, float *massFlux, int32_t nMassFlux,
                                                   float *su, int32_t nSu, float *uBoundary, int32_t nUBoundary,
                                                   float *vBoundary, int32_t nVBoundary, float *wBoundary,
                                                   int32_t nWBoundary, float fact, int32_t solveU, int32_t solveV,
                                                   int32_t solveW, const float *flowFact, int32_t nFlowFact,
                                                   float *flowout2);
int cupcfd_gpu_flux_mass_dolfyn_region_loop_f32(cupcfd_gpu_mesh *mesh, float *flowFact, int32_t nFlowFact,
                                               const float *flowRegion, int32_t nFlowRegion, float flowIn);

/* ------------------------------------------------------------------------ */
/* device-resident calls (device pointers, internal numbering, async)        */
/* ------------------------------------------------------------------------ */
/* Layouts (internal numbering; T = double for F64, float for F32C):
 *   cell scalar     T[nCells]
 *   cell vector     T[3][nCells]   (x block, then y, then z)
 *   face scalar     T[nFaces]      (internal face order; boundary entries unused)
 *   boundary scalar T[nBoundaries] (reference boundary order)
 *   cell state      T[4][nCells]   (rho, u, v, w blocks) for F64,
 *                   float4[nCells] (rho, u, v, w interleaved) for F32C
 * stream: a cudaStream_t (NULL = the legacy default stream).
 * Every array is aligned to its element (the F32C state to 16 bytes);
 * misaligned pointers are rejected with CUPCFD_E_CONFIG_INVALID_VALUE.
 * F32C forward/adjoint calls whose arrays start on 16-byte boundaries (and,
 * for the adjoint, nCells a multiple of 4) run the staged kernels, which
 * fetch each 256-cell tile's contiguous ranges into shared memory with bulk
 * async copies; other pointers take the unstaged kernels. Results are
 * bit-identical either way. */

/* Reorders n-component cell data (component blocks of nCells, element type
 * src_size / dst_size bytes = 4 or 8, converting) between numberings.
 * src_stride/dst_stride are the byte distance between component blocks
 * (0 = packed). to_internal: reference -> internal, else internal -> reference. */
int cupcfd_gpu_dev_permute_cells(const cupcfd_gpu_mesh *mesh, int32_t to_internal, int32_t ncomp,
                                 const void *src, int32_t src_size, int64_t src_comp_stride,
                                 void *dst, int32_t dst_size, int64_t dst_comp_stride, void *stream);
int cupcfd_gpu_dev_permute_faces(const cupcfd_gpu_mesh *mesh, int32_t to_internal,
                                 const void *src, int32_t src_size, void *dst, int32_t dst_size, void *stream);

/* Gradient, nGradient iterations (1 = the benchmark setting). grad_o may be
 * NULL (then an internal buffer holds the previous iterate). */
int cupcfd_gpu_dev_gradient(cupcfd_gpu_mesh *mesh, int32_t precision, int32_t nGradient, int32_t sign_mode,
                            const void *phi, const void *phiB, void *grad, void *grad_o, void *stream);
/* Plain mass flux m_f = rho_f (u_f . S_f) on interior faces; boundary entries untouched. */
int cupcfd_gpu_dev_mass_plain(cupcfd_gpu_mesh *mesh, int32_t precision, const void *state, void *massFlux, void *stream);
/* Adjoints: gradient (nGradient = 1): gbar (cell vector) -> phiBar, phiBBar;
 * plain mass flux: mbar (face scalar) -> stateBar (cell state layout). */
int cupcfd_gpu_dev_gradient_adjoint(cupcfd_gpu_mesh *mesh, int32_t precision, int32_t sign_mode, const void *gbar,
                                    void *phiBar, void *phiBBar, void *stream);
int cupcfd_gpu_dev_mass_plain_adjoint(cupcfd_gpu_mesh *mesh, int32_t precision, const void *state, const void *mbar,
                                      void *stateBar, void *stream);
/* Fused forward of both face loops (nGradient = 1): one launch computes
 * grad (cell vector) and massFlux (face scalar, interior faces) from phi,
 * phiB and state. With gface and loss non-NULL it also reduces, in FP64 and
 * in a fixed order, L = sum_c V_c |grad_c|^2 + sum_{interior f} gface_f m_f
 * into loss (device double[1]). */
int cupcfd_gpu_dev_forward(cupcfd_gpu_mesh *mesh, int32_t precision, const void *phi, const void *phiB,
                           const void *state, const void *gface, void *grad, void *massFlux, double *loss, void *stream);
/* Adjoint of that loss in one launch (the transposed gather): from grad,
 * state and gface it writes phiBar (cell scalar), phiBBar (boundary scalar)
 * and stateBar (cell state layout). */
int cupcfd_gpu_dev_adjoint(cupcfd_gpu_mesh *mesh, int32_t precision, const void *grad, const void *state,
                           const void *gface, void *phiBar, void *phiBBar, void *stateBar, void *stream);
/* The forward above without any allocation. No counterpart in the
 * reference. For callers that cannot allocate device memory when they run
 * the forward (a solver that reserves its whole memory budget at start-up,
 * or code running inside another runtime that owns the device allocator):
 * the loss partials live in a fixed array inside the library instead of the
 * mesh's scratch pool, and the call makes no cudaMalloc/cudaFree or other
 * allocating call. Same arguments and results as cupcfd_gpu_dev_forward.
 * Limits: the array holds 524,288 partials (one per warp: 4 MiB per GPU that
 * loads the library, held until exit), so with a loss the mesh may have at most
 * 16,777,216 cells; larger meshes return CUPCFD_E_ARRAY_SIZE_MISMATCH. All
 * calls share the array: calls whose kernels overlap on the GPU race. The
 * first call on a device sets up the array's address with that device
 * current; make it before any stream capture. The call runs on the mesh's
 * device and gives the caller's current device back before it returns.
 * Errors are reported by status code only (cupcfd_gpu_last_error is not
 * updated). */
int cupcfd_gpu_dev_forward_noalloc(cupcfd_gpu_mesh *mesh, int32_t precision, const void *phi, const void *phiB,
                                   const void *state, const void *gface, void *grad, void *massFlux, double *loss,
                                   void *stream);
/* Fused forward + adjoint of the benchmark loss (see cupcfd_gpu_forward_adjoint):
 * two launches over the mesh. Outputs grad, massFlux, phiBar, phiBBar,
 * stateBar; loss (device double[1], may be NULL) reduced in FP64. */
int cupcfd_gpu_dev_forward_adjoint(cupcfd_gpu_mesh *mesh, int32_t precision, const void *phi, const void *phiB,
                                   const void *state, const void *gface, void *grad, void *massFlux,
                                   void *phiBar, void *phiBBar, void *stateBar, double *loss, void *stream);

/* FP64 error norms of a against b (device arrays of n elements each,
 * a_size/b_size = 4 or 8 bytes): out[0] = max |a-b|, out[1] = max |b|,
 * out[2] = sum (a-b)^2, out[3] = sum b^2, out[4] = max |a-b| / max(|b|, floor).
 * out is a host double[5]; the call synchronises the stream. */
int cupcfd_gpu_dev_error_norms(const void *a, int32_t a_size, const void *b, int32_t b_size, int64_t n, double floor,
                               double *out, void *stream);

/* The boundary / region loops on device arrays (same semantics as the
 * host-buffer calls above): massFlux in internal face order, su in internal
 * cell order, boundary arrays by boundary id and region arrays by region id;
 * every scalar (flowin, ratearea, flowout, flowout2, flowIn) is a device
 * double, so the loops chain without synchronising. */
int cupcfd_gpu_dev_boundary_loop1(cupcfd_gpu_mesh *mesh, const double *massFlux, double *flowin, void *stream);
int cupcfd_gpu_dev_boundary_loop2(cupcfd_gpu_mesh *mesh, const double *massFlux, double *flowRegion, double *flowout,
                                  void *stream);
int cupcfd_gpu_dev_boundary_loop3(cupcfd_gpu_mesh *mesh, const double *flowin, double *ratearea, void *stream);
int cupcfd_gpu_dev_boundary_loop4(cupcfd_gpu_mesh *mesh, double *massFlux, double *uBoundary, double *vBoundary,
                                  double *wBoundary, const double *denBoundary, const double *ratearea,
                                  double *flowout, void *stream);
int cupcfd_gpu_dev_boundary_loop5(cupcfd_gpu_mesh *mesh, double *massFlux, double *su, double *uBoundary,
                                  double *vBoundary, double *wBoundary, double fact, int32_t solveU, int32_t solveV,
                                  int32_t solveW, const double *flowFact, double *flowout2, void *stream);
int cupcfd_gpu_dev_region_loop(cupcfd_gpu_mesh *mesh, double *flowFact, const double *flowRegion,
                               const double *flowIn, void *stream);

/* ------------------------------------------------------------------------ */
/* momentum face loop (UVWKernels.h:45-92, UVWKernels.ipp:38-544), FP64     */
/* ------------------------------------------------------------------------ */

/* Mesh state the momentum loops read and write. rlencos[nFaces] (reference
 * face order; replaces setFaceRLencos/getFaceRLencos,
 * UnstructuredMeshInterface.h:757-770) and distance[nBoundaries] (replaces
 * getBoundaryDistance, :1225-1238) are zero until set, as on every mesh a
 * MeshSource builds (UnstructuredMeshInterface.ipp:1809-1810,
 * MeshStructGenSource.cpp:1251-1258); NULL resets to zero. The boundary shear
 * [3*nBoundaries] (get/setBoundaryShear, :1333-1346, :1527) and region force
 * tangents [3*nRegions] (get/setRegionForceTangent, :1909-1922, :2225) are
 * xyz-interleaved; `in` (may be NULL) is written first, then `out` (may be
 * NULL) read. Both start at zero; cupcfd_gpu_mesh_set_regions zeroes the
 * force tangents. */
int cupcfd_gpu_mesh_set_face_rlencos(cupcfd_gpu_mesh *mesh, const double *rlencos, int32_t nFaces);
int cupcfd_gpu_mesh_set_boundary_distance(cupcfd_gpu_mesh *mesh, const double *distance, int32_t nBoundaries);
int cupcfd_gpu_mesh_boundary_shear(cupcfd_gpu_mesh *mesh, const double *in, double *out, int32_t nBoundaries);
int cupcfd_gpu_mesh_region_force_tangent(cupcfd_gpu_mesh *mesh, const double *in, double *out, int32_t nRegions);

/* cupcfd::fvm::FluxUVWDolfynFaceLoop1 (UVWKernels.h:45-67): host buffers in
 * the reference's numbering, same parameters in the same order; dudx/dvdx/
 * dwdx are vec3 views of the EuclideanVector<double,3> arrays. Updates
 * massFlux (outlet faces: negative fluxes become `small`), rFace (interior
 * faces), su/sv/sw, au/av/aw, u/v/wBoundary and the mesh's boundary shear
 * (wall faces) bit-identically to the reference. The reference carries
 * uFace/vFace/wFace and visFace from one face to the next in label order
 * (declared outside its face loop, UVWKernels.ipp:74-75: interior faces read
 * the values of the last inlet or outlet face before them, symmetry faces the
 * visFace of the last interior, inlet or outlet face); where the reference
 * reads them before any face set them (uninitialised there) they are zero
 * here. Arrays shorter than the mesh return E_INVALID_INDEX. */
int cupcfd_gpu_flux_uvw_dolfyn_face_loop1(
    cupcfd_gpu_mesh *mesh, double gammaBlend, double small, const double *uCell, int32_t nUCell,
    const double *vCell, int32_t nVCell, const double *wCell, int32_t nWCell, double *uBoundary, int32_t nUBoundary,
    double *vBoundary, int32_t nVBoundary, double *wBoundary, int32_t nWBoundary, const double *visEffCell,
    int32_t nVisEffCell, const double *visEffBoundary, int32_t nVisEffBoundary, double *massFlux, int32_t nMassFlux,
    cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx, int32_t nDwdx,
    double *rFace, int32_t nRFace, double *su, int32_t nSu, double *sv, int32_t nSv, double *sw, int32_t nSw,
    double *au, int32_t nAu, double *av, int32_t nAv, double *aw, int32_t nAw);
/* The same loop of the reference's T = float instantiation: float arrays,
 * EuclideanVector<float,3> views, the float build's arithmetic on the mesh's
 * FP32 geometry (exact for a mesh uploaded from float arrays), results bit
 * for bit those of the reference's float build. The mesh must have
 * CUPCFD_PREC_F32C geometry. */
int cupcfd_gpu_flux_uvw_dolfyn_face_loop1_f32(
    cupcfd_gpu_mesh *mesh, float gammaBlend, float small, const float *uCell, int32_t nUCell,
    const float *vCell, int32_t nVCell, const float *wCell, int32_t nWCell, float *uBoundary, int32_t nUBoundary,
    float *vBoundary, int32_t nVBoundary, float *wBoundary, int32_t nWBoundary, const float *visEffCell,
    int32_t nVisEffCell, const float *visEffBoundary, int32_t nVisEffBoundary, float *massFlux, int32_t nMassFlux,
    cupcfd_vec3_view dudx, int32_t nDudx, cupcfd_vec3_view dvdx, int32_t nDvdx, cupcfd_vec3_view dwdx, int32_t nDwdx,
    float *rFace, int32_t nRFace, float *su, int32_t nSu, float *sv, int32_t nSv, float *sw, int32_t nSw,
    float *au, int32_t nAu, float *av, int32_t nAv, float *aw, int32_t nAw);
/* FluxUVWDolfynRegionLoop1 (UVWKernels.ipp:517-524): force tangents = 0.
 * FluxUVWDolfynBndsLoop1 (UVWKernels.ipp:527-544): each wall boundary adds
 * its shear onto its region's force tangent, in boundary order; in float on
 * a mesh created from float arrays (real_size 4, the reference's T = float
 * instantiation), in double otherwise. The shears and tangents are kept in
 * double either way (a float mesh's values exactly). */
int cupcfd_gpu_flux_uvw_dolfyn_region_loop1(cupcfd_gpu_mesh *mesh);
int cupcfd_gpu_flux_uvw_dolfyn_bnds_loop1(cupcfd_gpu_mesh *mesh);

/* The same on device arrays in the mesh's internal numbering and a caller
 * stream: cell arrays [nCells], grads = 9 blocks of leading dimension ldg
 * (dudx x, y, z, dvdx x, y, z, dwdx x, y, z), face arrays [nFaces] and rFace
 * [2*nFaces] in internal face order, boundary arrays by boundary id. */
int cupcfd_gpu_dev_uvw_face_loop1(cupcfd_gpu_mesh *mesh, double gammaBlend, double small, const double *uCell,
                                  const double *vCell, const double *wCell, double *uBoundary, double *vBoundary,
                                  double *wBoundary, const double *visEffCell, const double *visEffBoundary,
                                  double *massFlux, const double *grads, int64_t ldg, double *rFace, double *su,
                                  double *sv, double *sw, double *au, double *av, double *aw, void *stream);
int cupcfd_gpu_dev_uvw_region_loop1(cupcfd_gpu_mesh *mesh, void *stream);
int cupcfd_gpu_dev_uvw_bnds_loop1(cupcfd_gpu_mesh *mesh, void *stream);

/* ------------------------------------------------------------------------ */
/* halo exchange of a mesh split across ranks                               */
/* ------------------------------------------------------------------------ */

/* Pack / unpack halves of a two-sided halo exchange (replace
 * ExchangePatternTwoSidedNonBlocking::packSendBuffer / unpackRecvBuffer,
 * src/comm/implementation/component/ExchangePatternTwoSidedNonBlocking.cpp:129-170),
 * on device arrays and a caller stream; the transfer between them is the
 * caller's (NCCL send / recv). Element-major buffers:
 *   pack:   dst[i*ncomp + c]  = src[c*ld + idx[i]]   (i < n, c < ncomp)
 *   unpack: dst[c*ld + idx[i]] = src[i*ncomp + c]
 * elemSize 4, 8 or 16 (a float4 state record as one element); idx[n] are
 * cells in the mesh's internal numbering (device int32). */
int cupcfd_gpu_dev_halo_pack(const void *src, int32_t elemSize, int32_t ncomp, int64_t ld, const int32_t *idx,
                             int32_t n, void *dst, void *stream);
int cupcfd_gpu_dev_halo_unpack(const void *src, int32_t elemSize, int32_t ncomp, int32_t n, const int32_t *idx,
                               void *dst, int64_t ld, void *stream);

/* The same for up to 8 fields at once, one launch per call (the fields of
 * one exchange share the index list): field k moves between fields[k].field
 * (ncomp components ld apart, elemSize 4, 8 or 16 bytes) and its own
 * element-major buffer fields[k].buffer, as the single-field calls do. */
typedef struct cupcfd_halo_field {
    void *field;
    int32_t elemSize, ncomp;
    int64_t ld;
    void *buffer;
} cupcfd_halo_field;
int cupcfd_gpu_dev_halo_pack_fields(const cupcfd_halo_field *fields, int32_t nFields, const int32_t *idx, int32_t n,
                                    void *stream);
int cupcfd_gpu_dev_halo_unpack_fields(const cupcfd_halo_field *fields, int32_t nFields, const int32_t *idx, int32_t n,
                                      void *stream);

/* Number of kernels this library launched since load (all threads). */
int64_t cupcfd_gpu_launch_count(void);

/* Device timers for measurement (no counterpart in the reference, whose
 * benchmarks time whole calls on the host): while enabled, every kernel
 * launch of the cupcfd_gpu_dev_forward / _adjoint / _forward_adjoint calls
 * is bracketed by two CUDA events on the stream it is launched on.
 * cupcfd_gpu_timing_read waits for the recorded events and returns, for up
 * to `capacity` kernels, the kernel name (NUL-terminated, at most 63
 * characters, in names[64 * i]), its launch count and its summed device
 * milliseconds since the previous read; *count receives the number of
 * kernels. Reading clears the record. Disabled by default. */
int cupcfd_gpu_timing_enable(int32_t on);
int cupcfd_gpu_timing_read(int32_t capacity, char *names, int64_t *launches, double *ms, int32_t *count);

#ifdef __cplusplus
}
#endif
#endif
