/*
 * C entry points over the reference's OWN CPU code, compiled unchanged from
 * the reference source tree into oracle/_ref/libcupcfd_ref.so by
 * oracle/Makefile (target "ref").
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the shipped library links this. It is
 * used (a) in this container to validate the plain-C restatement in
 * oracle/cupcfd_oracle.c, and (b) as the timed CPU reference arm.
 *
 * Wrapped reference code:
 *   - cupcfd::fvm::GradientPhiGaussDolfyn   include/fvm/implementation/component/GradientKernels.ipp:38-136
 *   - cupcfd::fvm::FluxMassDolfynFaceLoop   include/fvm/implementation/component/MassKernels.ipp:36-309
 *   - the mass boundary / region loops       MassKernels.ipp:311-554
 *   - cupcfd::fvm::FluxUVWDolfynFaceLoop1 / RegionLoop1 / BndsLoop1
 *                                            include/fvm/implementation/component/UVWKernels.ipp:38-544
 *   - MeshStructGenSource<int,double>       src/geometry/mesh/implementation/source/MeshStructGenSource.cpp:33-1277
 * The mesh the kernels see is the one-rank CupCfdSoAMesh that addData
 * (include/geometry/mesh/interface/component/UnstructuredMeshInterface.ipp:1464-1862)
 * builds from the generator: faces, boundaries and cells in ascending label
 * order, xpac = xnac = 0, every region RTYPE_DEFAULT.
 */
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>

#include "Error.h"
#include "EuclideanVector.h"
#include "EuclideanPoint.h"
#include "GradientKernels.h"
#include "MassKernels.h"
#include "UVWKernels.h"
#include "MeshStructGenSource.h"

namespace euc = cupcfd::geometry::euclidean;
namespace msh = cupcfd::geometry::mesh;

typedef msh::UnstructuredMeshInterface<int, int, double, int> RefMesh;

/* Error code values, exported so the tests can pin the C ABI's constants. */
extern "C" int ref_ecode_success() { return (int) cupcfd::error::E_SUCCESS; }
extern "C" int ref_ecode_invalid_index() { return (int) cupcfd::error::E_INVALID_INDEX; }
extern "C" int ref_ecode_array_size_mismatch() { return (int) cupcfd::error::E_ARRAY_SIZE_MISMATCH; }
extern "C" int ref_ecode_error() { return (int) cupcfd::error::E_ERROR; }
extern "C" int ref_ecode_null_ptr() { return (int) cupcfd::error::E_NULL_PTR; }
extern "C" int ref_ecode_not_implemented() { return (int) cupcfd::error::E_NOT_IMPLEMENTED; }
extern "C" int ref_ecode_file_missing() { return (int) cupcfd::error::E_FILE_MISSING; }
extern "C" int ref_ecode_invalid_file_format() { return (int) cupcfd::error::E_INVALID_FILE_FORMAT; }
extern "C" int ref_ecode_config_opt_not_found() { return (int) cupcfd::error::E_CONFIG_OPT_NOT_FOUND; }
extern "C" int ref_sizeof_euclidean_vector_f64() { return (int) sizeof(euc::EuclideanVector<double,3>); }
extern "C" int ref_sizeof_euclidean_vector_f32() { return (int) sizeof(euc::EuclideanVector<float,3>); }
extern "C" int ref_offsetof_cmp_f64() {
	euc::EuclideanVector<double,3> v;
	return (int) ((char *) &v.cmp[0] - (char *) &v);
}

/* ---- structured generator ------------------------------------------------ */

extern "C" void ref_structgen_counts(int nx, int ny, int nz, int * nCells, int * nFaces, int * nBnd, int * nVerts) {
	msh::MeshStructGenSource<int, double> src(nx, ny, nz, 0.0, 1.0, 0.0, 1.0, 0.0, 1.0);
	src.getCellCount(nCells);
	src.getFaceCount(nFaces);
	src.getBoundaryCount(nBnd);
	src.getVertexCount(nVerts);
}

/* Build every array the face loops read, for all labels in ascending order.
 * faceBnd[f] is the boundary label of f, or -1 for an interior face. */
extern "C" int ref_structgen_build(int nx, int ny, int nz,
                                   double xmin, double xmax, double ymin, double ymax, double zmin, double zmax,
                                   int * faceCell1, int * faceCell2, int * faceBnd,
                                   double * faceLambda, double * faceNorm, double * faceCenter, double * faceArea,
                                   double * cellCenter, double * cellVolume,
                                   int * cellFaceXAdj, int * cellFaceAdj,
                                   int * faceVert, double * vertCoords) {
	msh::MeshStructGenSource<int, double> src(nx, ny, nz, xmin, xmax, ymin, ymax, zmin, zmax);
	int nC, nF, nB, nV;
	src.getCellCount(&nC);
	src.getFaceCount(&nF);
	src.getBoundaryCount(&nB);
	src.getVertexCount(&nV);
	cupcfd::error::eCodes st;

	std::vector<int> cl(nC), fl(nF), vl(nV);
	for (int i = 0; i < nC; i++) cl[i] = i;
	for (int i = 0; i < nF; i++) fl[i] = i;
	for (int i = 0; i < nV; i++) vl[i] = i;

	bool * isB = (bool *) malloc(sizeof(bool) * nF);
	st = src.getFaceIsBoundary(isB, nF, fl.data(), nF);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;
	st = src.getFaceCell1Labels(faceCell1, nF, fl.data(), nF);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;

	std::vector<int> interior, boundary;
	for (int f = 0; f < nF; f++) (isB[f] ? boundary : interior).push_back(f);
	std::vector<int> c2(interior.size()), bl(boundary.size());
	if (!interior.empty()) {
		st = src.getFaceCell2Labels(c2.data(), (int) interior.size(), interior.data(), (int) interior.size());
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
	}
	if (!boundary.empty()) {
		st = src.getFaceBoundaryLabels(bl.data(), (int) boundary.size(), boundary.data(), (int) boundary.size());
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
	}
	for (int f = 0; f < nF; f++) { faceCell2[f] = -1; faceBnd[f] = -1; }
	for (size_t k = 0; k < interior.size(); k++) faceCell2[interior[k]] = c2[k];
	for (size_t k = 0; k < boundary.size(); k++) faceBnd[boundary[k]] = bl[k];
	free(isB);

	st = src.getFaceLambda(faceLambda, nF, fl.data(), nF);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;
	st = src.getFaceArea(faceArea, nF, fl.data(), nF);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;

	std::vector<euc::EuclideanVector<double,3>> nrm(nF);
	st = src.getFaceNormal(nrm.data(), nF, fl.data(), nF);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;
	std::vector<euc::EuclideanPoint<double,3>> fc(nF);
	st = src.getFaceCenter(fc.data(), nF, fl.data(), nF);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;
	for (int f = 0; f < nF; f++) {
		for (int d = 0; d < 3; d++) {
			faceNorm[3*f+d] = nrm[f].cmp[d];
			faceCenter[3*f+d] = fc[f].cmp[d];
		}
	}

	std::vector<euc::EuclideanPoint<double,3>> cc(nC);
	st = src.getCellCenter(cc.data(), nC, cl.data(), nC);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;
	st = src.getCellVolume(cellVolume, nC, cl.data(), nC);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;
	for (int c = 0; c < nC; c++)
		for (int d = 0; d < 3; d++) cellCenter[3*c+d] = cc[c].cmp[d];

	if (cellFaceXAdj && cellFaceAdj) {
		st = src.getCellFaceLabels(cellFaceXAdj, nC + 1, cellFaceAdj, 6 * nC, cl.data(), nC);
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
	}
	if (faceVert) {
		std::vector<int> xadj(nF + 1);
		st = src.getFaceVerticesLabelsCSR(xadj.data(), nF + 1, faceVert, 4 * nF, fl.data(), nF);
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
	}
	if (vertCoords) {
		std::vector<euc::EuclideanPoint<double,3>> vc(nV);
		st = src.getVertexCoords(vc.data(), nV, vl.data(), nV);
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
		for (int v = 0; v < nV; v++)
			for (int d = 0; d < 3; d++) vertCoords[3*v+d] = vc[v].cmp[d];
	}
	return (int) cupcfd::error::E_SUCCESS;
}

/* ---- kernel context --------------------------------------------------------
 * Holds a shim mesh over caller-owned arrays plus the reference's vptr'd
 * EuclideanVector field arrays, so that timing covers only the kernel call,
 * as the reference's TreeTimer block does (src/benchmarks/.../BenchmarkKernels.cpp:166-186). */
struct RefCtx {
	RefMesh mesh;
	int nC, nF, nB, nR;
	std::vector<euc::EuclideanVector<double,3>> g, go;
	std::vector<euc::EuclideanVector<double,3>> dudx, dvdx, dwdx, dpdx;
	std::vector<int> boundaryFace;   /* getBoundaryFaceID: faceBnd inverted */
	std::vector<double> splvl;       /* getRegionSplvl (ref_ctx_set_splvl) */
	std::vector<double> rlencos, bdist, shear, ftan;   /* momentum-loop mesh state, zero until set */
};

extern "C" void * ref_ctx_create(int nCells, int nFaces, int nBnd, int nRegions,
                                 const int * faceCell1, const int * faceCell2, const int * faceBnd,
                                 const double * faceLambda, const double * faceNorm, const double * faceCenter,
                                 const double * faceArea, const double * faceXpac, const double * faceXnac,
                                 const double * cellCenter, const double * cellVolume,
                                 const int * boundaryRegion, const int * regionType,
                                 const double * regionUVW, const double * regionDen) {
	RefCtx * c = new RefCtx();
	c->nC = nCells; c->nF = nFaces; c->nB = nBnd; c->nR = nRegions;
	c->mesh.properties.lOCells = nCells;
	c->mesh.properties.lGhCells = 0;
	c->mesh.properties.lTCells = nCells;
	c->mesh.properties.lFaces = nFaces;
	c->mesh.properties.lBoundaries = nBnd;
	c->mesh.properties.lRegions = nRegions;
	c->mesh.a.faceCell1 = faceCell1;
	c->mesh.a.faceCell2 = faceCell2;
	c->mesh.a.faceBoundary = faceBnd;
	c->mesh.a.faceLambda = faceLambda;
	c->mesh.a.faceNorm = faceNorm;
	c->mesh.a.faceCenter = faceCenter;
	c->mesh.a.faceArea = faceArea;
	c->mesh.a.faceXpac = faceXpac;
	c->mesh.a.faceXnac = faceXnac;
	c->mesh.a.cellCenter = cellCenter;
	c->mesh.a.cellVolume = cellVolume;
	c->mesh.a.boundaryRegion = boundaryRegion;
	c->mesh.a.regionType = regionType;
	c->mesh.a.regionUVW = regionUVW;
	c->mesh.a.regionDen = regionDen;
	c->boundaryFace.assign(nBnd > 0 ? nBnd : 1, -1);
	for (int f = 0; f < nFaces; f++)
		if (faceBnd[f] > -1) c->boundaryFace[faceBnd[f]] = f;
	c->mesh.a.boundaryFace = c->boundaryFace.data();
	c->splvl.assign(nRegions > 0 ? nRegions : 1, 0.0);
	c->mesh.a.regionSplvl = c->splvl.data();
	c->rlencos.assign(nFaces > 0 ? nFaces : 1, 0.0);
	c->bdist.assign(nBnd > 0 ? nBnd : 1, 0.0);
	c->shear.assign(3 * (nBnd > 0 ? nBnd : 1), 0.0);
	c->ftan.assign(3 * (nRegions > 0 ? nRegions : 1), 0.0);
	c->mesh.a.faceRLencos = c->rlencos.data();
	c->mesh.a.boundaryDistance = c->bdist.data();
	c->mesh.a.boundaryShear = c->shear.data();
	c->mesh.a.regionForceTangent = c->ftan.data();
	c->g.resize(nCells);
	c->go.resize(nCells);
	return c;
}

extern "C" void ref_ctx_destroy(void * p) { delete (RefCtx *) p; }

static void unpackVec(const std::vector<euc::EuclideanVector<double,3>> & v, double * out) {
	for (size_t i = 0; i < v.size(); i++)
		for (int d = 0; d < 3; d++) out[3*i+d] = v[i].cmp[d];
}
static void packVec(std::vector<euc::EuclideanVector<double,3>> & v, const double * in, int n) {
	v.resize(n);
	for (int i = 0; i < n; i++)
		for (int d = 0; d < 3; d++) v[i].cmp[d] = in[3*i+d];
}

/* Runs GradientPhiGaussDolfyn `reps` times; per-call seconds go to secs[reps]
 * (may be NULL). Outputs are the last call's dPhidxCell / dPhidxoCell. */
extern "C" int ref_gradient_phi_gauss(void * p, int nGradient, double * phi, int nPhi, double * phiB, int nPhiB,
                                      double * dPhidx, double * dPhidxo, int reps, double * secs) {
	RefCtx * c = (RefCtx *) p;
	cupcfd::error::eCodes st = cupcfd::error::E_SUCCESS;
	for (int r = 0; r < reps; r++) {
		auto t0 = std::chrono::steady_clock::now();
		st = cupcfd::fvm::GradientPhiGaussDolfyn(c->mesh, nGradient, phi, nPhi, phiB, nPhiB,
		                                         c->g.data(), c->nC, c->go.data(), c->nC);
		auto t1 = std::chrono::steady_clock::now();
		if (secs) secs[r] = std::chrono::duration<double>(t1 - t0).count();
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
	}
	if (dPhidx) unpackVec(c->g, dPhidx);
	if (dPhidxo) unpackVec(c->go, dPhidxo);
	return (int) st;
}

/* GradientPhiGaussDolfyn of the reference's T=float instantiation
 * (BenchmarkKernels.cpp:1134-1138 instantiates the kernels for float and
 * double meshes) on a float mesh given by its arrays; dPhidx / dPhidxo get
 * the components [3*nCells]. Only the getters the gradient calls are set. */
typedef msh::UnstructuredMeshInterface<int, int, float, int> RefMeshF;
extern "C" int ref_gradient_phi_gauss_f32(int nCells, int nFaces, int nBnd, const int * faceCell1,
                                          const int * faceCell2, const int * faceBnd, const float * faceLambda,
                                          const float * faceNorm, const float * faceCenter,
                                          const float * cellCenter, const float * cellVolume, int nGradient,
                                          float * phi, float * phiB, float * dPhidx, float * dPhidxo) {
	RefMeshF mesh;
	mesh.properties.lOCells = nCells;
	mesh.properties.lGhCells = 0;
	mesh.properties.lTCells = nCells;
	mesh.properties.lFaces = nFaces;
	mesh.properties.lBoundaries = nBnd;
	mesh.properties.lRegions = 1;
	mesh.a = {};
	mesh.a.faceCell1 = faceCell1;
	mesh.a.faceCell2 = faceCell2;
	mesh.a.faceBoundary = faceBnd;
	mesh.a.faceLambda = faceLambda;
	mesh.a.faceNorm = faceNorm;
	mesh.a.faceCenter = faceCenter;
	mesh.a.cellCenter = cellCenter;
	mesh.a.cellVolume = cellVolume;
	std::vector<euc::EuclideanVector<float,3>> g(nCells), go(nCells);
	cupcfd::error::eCodes st = cupcfd::fvm::GradientPhiGaussDolfyn(mesh, nGradient, phi, nCells, phiB, nBnd,
	                                                               g.data(), nCells, go.data(), nCells);
	for (int i = 0; i < nCells; i++)
		for (int d = 0; d < 3; d++) {
			dPhidx[3*i+d] = g[i].cmp[d];
			dPhidxo[3*i+d] = go[i].cmp[d];
		}
	return (int) st;
}

/* FluxMassDolfynFaceLoop of the reference's T=float instantiation on a float
 * mesh given by its arrays (xyz-interleaved vectors), regions included;
 * vector fields [3*nCells]; in/out arrays updated in place as the reference
 * does. */
extern "C" int ref_flux_mass_face_loop_f32(int nCells, int nFaces, int nBnd, int nRegions, const int * faceCell1,
                                           const int * faceCell2, const int * faceBnd, const float * faceLambda,
                                           const float * faceNorm, const float * faceCenter, const float * faceArea,
                                           const float * faceXpac, const float * faceXnac, const float * cellCenter,
                                           const float * cellVolume, const int * bndRegion, const int * regionType,
                                           const float * regionUVW, const float * regionDen,
                                           const float * dudx, const float * dvdx, const float * dwdx, const float * dpdx,
                                           float * den, float * denB, float * u, float * v, float * w,
                                           float * massFlux, float * pr, float * ar, float * su, float * rface,
                                           float small, int * icinl, int * icout, int * icsym, int * icwal,
                                           int solveTurbEnergy, int solveTurbDiss, int solveVisc, int solveEnthalpy,
                                           float * teC, float * teB, float * edC, float * edB,
                                           float * visC, float * visB, float * tC, float * tB) {
	RefMeshF mesh;
	mesh.properties.lOCells = nCells;
	mesh.properties.lGhCells = 0;
	mesh.properties.lTCells = nCells;
	mesh.properties.lFaces = nFaces;
	mesh.properties.lBoundaries = nBnd;
	mesh.properties.lRegions = nRegions;
	mesh.a = {};
	mesh.a.faceCell1 = faceCell1;
	mesh.a.faceCell2 = faceCell2;
	mesh.a.faceBoundary = faceBnd;
	mesh.a.faceLambda = faceLambda;
	mesh.a.faceNorm = faceNorm;
	mesh.a.faceCenter = faceCenter;
	mesh.a.faceArea = faceArea;
	mesh.a.faceXpac = faceXpac;
	mesh.a.faceXnac = faceXnac;
	mesh.a.cellCenter = cellCenter;
	mesh.a.cellVolume = cellVolume;
	mesh.a.boundaryRegion = bndRegion;
	mesh.a.regionType = regionType;
	mesh.a.regionUVW = regionUVW;
	mesh.a.regionDen = regionDen;
	std::vector<euc::EuclideanVector<float,3>> gu(nCells), gv(nCells), gw(nCells), gp(nCells);
	for (int i = 0; i < nCells; i++)
		for (int d = 0; d < 3; d++) {
			gu[i].cmp[d] = dudx[3*i+d]; gv[i].cmp[d] = dvdx[3*i+d];
			gw[i].cmp[d] = dwdx[3*i+d]; gp[i].cmp[d] = dpdx[3*i+d];
		}
	return (int) cupcfd::fvm::FluxMassDolfynFaceLoop(mesh,
		gu.data(), nCells, gv.data(), nCells, gw.data(), nCells, gp.data(), nCells,
		den, nCells, denB, nBnd, u, nCells, v, nCells, w, nCells, massFlux, nFaces, pr, nCells, ar, nCells, su, nCells,
		rface, 2 * nFaces, small, icinl, icout, icsym, icwal,
		solveTurbEnergy != 0, solveTurbDiss != 0, solveVisc != 0, solveEnthalpy != 0,
		teC, nCells, teB, nBnd, edC, nCells, edB, nBnd, visC, nCells, visB, nBnd, tC, nCells, tB, nBnd);
}

/* Runs FluxMassDolfynFaceLoop `reps` times with the reference's full
 * argument list. Vector fields are xyz-interleaved [3*nCells]. The arrays
 * massFlux, su, rface, denB and the te/ed/viseff/t boundary arrays are
 * updated in place exactly as the reference does. */
extern "C" int ref_flux_mass_face_loop(void * p,
                                       const double * dudx, const double * dvdx, const double * dwdx, const double * dpdx,
                                       double * den, double * denB, double * u, double * v, double * w,
                                       double * massFlux, double * pr, double * ar, double * su, double * rface,
                                       double small, int * icinl, int * icout, int * icsym, int * icwal,
                                       int solveTurbEnergy, int solveTurbDiss, int solveVisc, int solveEnthalpy,
                                       double * teC, double * teB, double * edC, double * edB,
                                       double * visC, double * visB, double * tC, double * tB,
                                       int reps, double * secs) {
	RefCtx * c = (RefCtx *) p;
	int nC = c->nC, nF = c->nF, nB = c->nB;
	packVec(c->dudx, dudx, nC);
	packVec(c->dvdx, dvdx, nC);
	packVec(c->dwdx, dwdx, nC);
	packVec(c->dpdx, dpdx, nC);
	cupcfd::error::eCodes st = cupcfd::error::E_SUCCESS;
	for (int r = 0; r < reps; r++) {
		auto t0 = std::chrono::steady_clock::now();
		st = cupcfd::fvm::FluxMassDolfynFaceLoop(c->mesh,
			c->dudx.data(), nC, c->dvdx.data(), nC, c->dwdx.data(), nC, c->dpdx.data(), nC,
			den, nC, denB, nB, u, nC, v, nC, w, nC, massFlux, nF, pr, nC, ar, nC, su, nC, rface, 2 * nF,
			small, icinl, icout, icsym, icwal,
			solveTurbEnergy != 0, solveTurbDiss != 0, solveVisc != 0, solveEnthalpy != 0,
			teC, nC, teB, nB, edC, nC, edB, nB, visC, nC, visB, nB, tC, nC, tB, nB);
		auto t1 = std::chrono::steady_clock::now();
		if (secs) secs[r] = std::chrono::duration<double>(t1 - t0).count();
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
	}
	return (int) st;
}

/* ---- boundary / region loops (MassKernels.ipp:311-554), called unchanged ---- */
extern "C" void ref_ctx_set_splvl(void * p, const double * splvl) {
	RefCtx * c = (RefCtx *) p;
	for (int r = 0; r < c->nR; r++) c->splvl[r] = splvl[r];
}

extern "C" int ref_boundary_loop1(void * p, double * massFlux, double * flowin) {
	RefCtx * c = (RefCtx *) p;
	return (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop1(c->mesh, massFlux, c->nF, flowin);
}

extern "C" int ref_boundary_loop2(void * p, double * massFlux, double * flowRegion, double * flowout) {
	RefCtx * c = (RefCtx *) p;
	return (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop2(c->mesh, massFlux, c->nF, flowRegion, c->nR, flowout);
}

extern "C" int ref_boundary_loop3(void * p, double flowin, double * ratearea) {
	RefCtx * c = (RefCtx *) p;
	return (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop3(c->mesh, flowin, ratearea);
}

extern "C" int ref_boundary_loop4(void * p, double * massFlux, double * uB, double * vB, double * wB, double * denB,
                                  double ratearea, double * flowout) {
	RefCtx * c = (RefCtx *) p;
	return (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop4(c->mesh, massFlux, c->nF, uB, c->nB, vB, c->nB, wB, c->nB,
	                                                        denB, c->nB, ratearea, flowout);
}

extern "C" int ref_boundary_loop5(void * p, double * massFlux, double * su, double * uB, double * vB, double * wB,
                                  double fact, int solveU, int solveV, int solveW, double * flowFact, double * flowout2) {
	RefCtx * c = (RefCtx *) p;
	return (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop5(c->mesh, massFlux, c->nF, su, c->nC, uB, c->nB, vB, c->nB,
	                                                        wB, c->nB, fact, solveU != 0, solveV != 0, solveW != 0,
	                                                        flowFact, c->nR, flowout2);
}

extern "C" int ref_region_loop(void * p, double * flowFact, double * flowRegion, double flowIn) {
	RefCtx * c = (RefCtx *) p;
	return (int) cupcfd::fvm::FluxMassDolfynRegionLoop(c->mesh, flowFact, c->nR, flowRegion, c->nR, flowIn);
}

/* The boundary-loop chain of a solver step (loops 1, 3, 4, 2, the region
 * loop, 5), `reps` times on the same arrays (updated in place, as the GPU
 * chain does); per-chain seconds go to secs[reps]. Timing only. */
extern "C" int ref_boundary_chain(void * p, double * massFlux, double * su, double * uB, double * vB, double * wB,
                                  double * denB, double * flowRegion, double * flowFact, int reps, double * secs) {
	RefCtx * c = (RefCtx *) p;
	int st = 0;
	for (int r = 0; r < reps; r++) {
		double flowin = 0.0, ratearea = 0.0, flowout = 0.0, flowout2 = 0.25, flowout4 = 0.0;
		auto t0 = std::chrono::steady_clock::now();
		st |= ref_boundary_loop1(p, massFlux, &flowin) - (int) cupcfd::error::E_SUCCESS;
		st |= ref_boundary_loop3(p, flowin, &ratearea) - (int) cupcfd::error::E_SUCCESS;
		st |= ref_boundary_loop4(p, massFlux, uB, vB, wB, denB, ratearea, &flowout4) - (int) cupcfd::error::E_SUCCESS;
		st |= ref_boundary_loop2(p, massFlux, flowRegion, &flowout) - (int) cupcfd::error::E_SUCCESS;
		st |= ref_region_loop(p, flowFact, flowRegion, flowin) - (int) cupcfd::error::E_SUCCESS;
		st |= ref_boundary_loop5(p, massFlux, su, uB, vB, wB, 1.3, 1, 1, 1, flowFact, &flowout2) -
		      (int) cupcfd::error::E_SUCCESS;
		auto t1 = std::chrono::steady_clock::now();
		if (secs) secs[r] = std::chrono::duration<double>(t1 - t0).count();
	}
	return st == 0 ? (int) cupcfd::error::E_SUCCESS : (int) cupcfd::error::E_ERROR;
}

/* The boundary-loop chain (loops 1, 3, 4, 2, the region loop, 5) of the
 * reference's T=float instantiation on a float mesh given by its arrays,
 * once, arrays updated in place; out[5] = flowin, ratearea, flowout (loop 4),
 * flowout (loop 2), flowout2 (from flowout2In). */
extern "C" int ref_boundary_chain_f32(int nCells, int nFaces, int nBnd, int nRegions, const int * faceCell1,
                                      const int * faceBnd, const float * faceNorm, const float * faceArea,
                                      const int * bndRegion, const int * regionType, const float * splvl,
                                      float * massFlux, float * su, float * uB, float * vB, float * wB,
                                      const float * denB, float * flowRegion, float * flowFact, float fact,
                                      int solveU, int solveV, int solveW, float flowout2In, float * out) {
	RefMeshF mesh;
	mesh.properties.lOCells = nCells;
	mesh.properties.lGhCells = 0;
	mesh.properties.lTCells = nCells;
	mesh.properties.lFaces = nFaces;
	mesh.properties.lBoundaries = nBnd;
	mesh.properties.lRegions = nRegions;
	mesh.a = {};
	mesh.a.faceCell1 = faceCell1;
	mesh.a.faceBoundary = faceBnd;
	mesh.a.faceNorm = faceNorm;
	mesh.a.faceArea = faceArea;
	mesh.a.boundaryRegion = bndRegion;
	mesh.a.regionType = regionType;
	mesh.a.regionSplvl = splvl;
	std::vector<int> bface(nBnd > 0 ? nBnd : 1, -1);
	for (int f = 0; f < nFaces; f++)
		if (faceBnd[f] > -1) bface[faceBnd[f]] = f;
	mesh.a.boundaryFace = bface.data();
	float flowin = 0.0f, ratearea = 0.0f, flowout4 = 0.0f, flowout = 0.0f, flowout2 = flowout2In;
	std::vector<float> den(denB, denB + nBnd);
	int st = 0;
	const int ok = (int) cupcfd::error::E_SUCCESS;
	st |= (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop1(mesh, massFlux, nFaces, &flowin) - ok;
	st |= (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop3(mesh, flowin, &ratearea) - ok;
	st |= (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop4(mesh, massFlux, nFaces, uB, nBnd, vB, nBnd, wB, nBnd,
	                                                       den.data(), nBnd, ratearea, &flowout4) - ok;
	st |= (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop2(mesh, massFlux, nFaces, flowRegion, nRegions, &flowout) - ok;
	st |= (int) cupcfd::fvm::FluxMassDolfynRegionLoop(mesh, flowFact, nRegions, flowRegion, nRegions, flowin) - ok;
	st |= (int) cupcfd::fvm::FluxMassDolfynBoundaryLoop5(mesh, massFlux, nFaces, su, nCells, uB, nBnd, vB, nBnd, wB,
	                                                       nBnd, fact, solveU != 0, solveV != 0, solveW != 0,
	                                                       flowFact, nRegions, &flowout2) - ok;
	out[0] = flowin; out[1] = ratearea; out[2] = flowout4; out[3] = flowout; out[4] = flowout2;
	return st == 0 ? ok : (int) cupcfd::error::E_ERROR;
}

/* ---- momentum loops (UVWKernels.ipp:38-544), called unchanged ---- */
extern "C" void ref_ctx_set_uvw_geometry(void * p, const double * rlencos, const double * bdist) {
	RefCtx * c = (RefCtx *) p;
	for (int f = 0; f < c->nF; f++) c->rlencos[f] = rlencos ? rlencos[f] : 0.0;
	for (int b = 0; b < c->nB; b++) c->bdist[b] = bdist ? bdist[b] : 0.0;
}

/* shear[3*nBnd] and forceTangent[3*nRegions] in / out (either may be NULL). */
extern "C" void ref_uvw_state(void * p, const double * shearIn, const double * ftanIn, double * shearOut, double * ftanOut) {
	RefCtx * c = (RefCtx *) p;
	if (shearIn) std::copy(shearIn, shearIn + 3 * c->nB, c->shear.begin());
	if (ftanIn) std::copy(ftanIn, ftanIn + 3 * c->nR, c->ftan.begin());
	if (shearOut) std::copy(c->shear.begin(), c->shear.begin() + 3 * c->nB, shearOut);
	if (ftanOut) std::copy(c->ftan.begin(), c->ftan.begin() + 3 * c->nR, ftanOut);
}

/* Runs FluxUVWDolfynFaceLoop1 `reps` times with the reference's argument
 * list; in/out arrays are updated in place as the reference does. */
extern "C" int ref_uvw_face_loop1(void * p, double gammaBlend, double small, double * u, double * v, double * w,
                                  double * uB, double * vB, double * wB, double * visC, double * visB,
                                  double * massFlux, const double * dudx, const double * dvdx, const double * dwdx,
                                  double * rFace, double * su, double * sv, double * sw, double * au, double * av,
                                  double * aw, int reps, double * secs) {
	RefCtx * c = (RefCtx *) p;
	int nC = c->nC, nF = c->nF, nB = c->nB;
	packVec(c->dudx, dudx, nC);
	packVec(c->dvdx, dvdx, nC);
	packVec(c->dwdx, dwdx, nC);
	cupcfd::error::eCodes st = cupcfd::error::E_SUCCESS;
	for (int r = 0; r < reps; r++) {
		auto t0 = std::chrono::steady_clock::now();
		st = cupcfd::fvm::FluxUVWDolfynFaceLoop1(c->mesh, gammaBlend, small, u, nC, v, nC, w, nC, uB, nB, vB, nB, wB, nB,
		                                          visC, nC, visB, nB, massFlux, nF, c->dudx.data(), nC, c->dvdx.data(), nC,
		                                          c->dwdx.data(), nC, rFace, 2 * nF, su, nC, sv, nC, sw, nC, au, nC,
		                                          av, nC, aw, nC);
		auto t1 = std::chrono::steady_clock::now();
		if (secs) secs[r] = std::chrono::duration<double>(t1 - t0).count();
		if (st != cupcfd::error::E_SUCCESS) return (int) st;
	}
	return (int) st;
}

extern "C" void ref_uvw_region_loop1(void * p) { cupcfd::fvm::FluxUVWDolfynRegionLoop1(((RefCtx *) p)->mesh); }
extern "C" void ref_uvw_bnds_loop1(void * p) { cupcfd::fvm::FluxUVWDolfynBndsLoop1(((RefCtx *) p)->mesh); }

/* The momentum loops of the reference's T=float instantiation on a float
 * mesh given by its arrays (xyz-interleaved vectors): FluxUVWDolfynFaceLoop1,
 * then FluxUVWDolfynRegionLoop1 and FluxUVWDolfynBndsLoop1 on the mesh's
 * shears and force tangents, which come back in shear[3*nBnd] and
 * ftan[3*nRegions] (ftan in: the tangents before the region loop zeroes
 * them, unused). In/out arrays updated in place as the reference does. */
extern "C" int ref_uvw_loops_f32(int nCells, int nFaces, int nBnd, int nRegions, const int * faceCell1,
                                 const int * faceCell2, const int * faceBnd, const float * faceLambda,
                                 const float * faceNorm, const float * faceCenter, const float * faceArea,
                                 const float * cellCenter, const float * cellVolume, const int * bndRegion,
                                 const int * regionType, const float * regionUVW, const float * regionDen,
                                 const float * rlencos, const float * bdist, float gammaBlend, float small,
                                 float * u, float * v, float * w, float * uB, float * vB, float * wB, float * visC,
                                 float * visB, float * massFlux, const float * dudx, const float * dvdx,
                                 const float * dwdx, float * rFace, float * su, float * sv, float * sw, float * au,
                                 float * av, float * aw, float * shear, float * ftan) {
	RefMeshF mesh;
	mesh.properties.lOCells = nCells;
	mesh.properties.lGhCells = 0;
	mesh.properties.lTCells = nCells;
	mesh.properties.lFaces = nFaces;
	mesh.properties.lBoundaries = nBnd;
	mesh.properties.lRegions = nRegions;
	mesh.a = {};
	mesh.a.faceCell1 = faceCell1;
	mesh.a.faceCell2 = faceCell2;
	mesh.a.faceBoundary = faceBnd;
	mesh.a.faceLambda = faceLambda;
	mesh.a.faceNorm = faceNorm;
	mesh.a.faceCenter = faceCenter;
	mesh.a.faceArea = faceArea;
	mesh.a.cellCenter = cellCenter;
	mesh.a.cellVolume = cellVolume;
	mesh.a.boundaryRegion = bndRegion;
	mesh.a.regionType = regionType;
	mesh.a.regionUVW = regionUVW;
	mesh.a.regionDen = regionDen;
	mesh.a.faceRLencos = rlencos;
	mesh.a.boundaryDistance = bdist;
	mesh.a.boundaryShear = shear;
	mesh.a.regionForceTangent = ftan;
	std::vector<euc::EuclideanVector<float,3>> gu(nCells), gv(nCells), gw(nCells);
	for (int i = 0; i < nCells; i++)
		for (int d = 0; d < 3; d++) {
			gu[i].cmp[d] = dudx[3*i+d]; gv[i].cmp[d] = dvdx[3*i+d]; gw[i].cmp[d] = dwdx[3*i+d];
		}
	cupcfd::error::eCodes st = cupcfd::fvm::FluxUVWDolfynFaceLoop1(mesh, gammaBlend, small, u, nCells, v, nCells,
		w, nCells, uB, nBnd, vB, nBnd, wB, nBnd, visC, nCells, visB, nBnd, massFlux, nFaces, gu.data(), nCells,
		gv.data(), nCells, gw.data(), nCells, rFace, 2 * nFaces, su, nCells, sv, nCells, sw, nCells, au, nCells,
		av, nCells, aw, nCells);
	if (st != cupcfd::error::E_SUCCESS) return (int) st;
	cupcfd::fvm::FluxUVWDolfynRegionLoop1(mesh);
	cupcfd::fvm::FluxUVWDolfynBndsLoop1(mesh);
	return (int) st;
}
