/*
 * Minimal stand-in for the reference's UnstructuredMeshInterface, exposing
 * exactly the getters that the reference kernels GradientPhiGaussDolfyn
 * (include/fvm/implementation/component/GradientKernels.ipp:39-136),
 * FluxMassDolfynFaceLoop (include/fvm/implementation/component/MassKernels.ipp:36-309),
 * the boundary / region loops (MassKernels.ipp:311-554) and the momentum
 * loops FluxUVWDolfynFaceLoop1 / RegionLoop1 / BndsLoop1
 * (include/fvm/implementation/component/UVWKernels.ipp:38-544) call, backed by
 * plain SoA arrays owned by the caller.
 *
 * TEST INFRASTRUCTURE ONLY: used to compile the reference's own kernel
 * templates, unchanged, into oracle/_ref/libcupcfd_ref.so. Getter names,
 * argument lists and return types follow
 * include/geometry/mesh/interface/component/UnstructuredMeshInterface.h
 * (lines 197-1949), so the reference templates compile without edits.
 */
#ifndef CUPCFD_ORACLE_SHIM_UNSTRUCTURED_MESH_INTERFACE_H
#define CUPCFD_ORACLE_SHIM_UNSTRUCTURED_MESH_INTERFACE_H

#include "EuclideanVector.h"
#include "EuclideanPoint.h"
#include "EuclideanVector3D.h"

namespace cupcfd
{
	namespace geometry
	{
		namespace mesh
		{
			/* Same enumerator order as the reference (UnstructuredMeshInterface.h:58-65). */
			enum RType
			{
				RTYPE_DEFAULT,
				RTYPE_INLET,
				RTYPE_OUTLET,
				RTYPE_SYMP,
				RTYPE_WALL
			};

			template <class I>
			struct ShimMeshProperties {
				I lOCells;
				I lGhCells;
				I lTCells;
				I lFaces;
				I lBoundaries;
				I lRegions;
			};

			/* Plain-array view of a mesh: every array indexed by local id. */
			template <class I, class T>
			struct ShimMeshArrays {
				const I * faceCell1;      /* [lFaces] */
				const I * faceCell2;      /* [lFaces], -1 on boundary faces */
				const I * faceBoundary;   /* [lFaces], -1 on interior faces */
				const T * faceLambda;     /* [lFaces] */
				const T * faceNorm;       /* [3*lFaces] xyz interleaved */
				const T * faceCenter;     /* [3*lFaces] */
				const T * faceArea;       /* [lFaces] */
				const T * faceXpac;       /* [3*lFaces] */
				const T * faceXnac;       /* [3*lFaces] */
				const T * cellCenter;     /* [3*lTCells] */
				const T * cellVolume;     /* [lTCells] */
				const I * boundaryRegion; /* [lBoundaries] */
				const int * regionType;   /* [lRegions] RType values */
				const T * regionUVW;      /* [3*lRegions] */
				const T * regionDen;      /* [lRegions] */
				const I * boundaryFace;   /* [lBoundaries] face of each boundary (getBoundaryFaceID) */
				const T * regionSplvl;    /* [lRegions] (getRegionSplvl) */
				const T * faceRLencos;    /* [lFaces] (getFaceRLencos) */
				const T * boundaryDistance; /* [lBoundaries] (getBoundaryDistance) */
				T * boundaryShear;        /* [3*lBoundaries] (get/setBoundaryShear) */
				T * regionForceTangent;   /* [3*lRegions] (get/setRegionForceTangent) */
			};

			template <class M, class I, class T, class L>
			class UnstructuredMeshInterface
			{
				public:
					ShimMeshProperties<I> properties;
					ShimMeshArrays<I, T> a;

					inline I getFaceCell1ID(I f) { return a.faceCell1[f]; }
					inline I getFaceCell2ID(I f) { return a.faceCell2[f]; }
					inline bool getFaceIsBoundary(I f) { return a.faceBoundary[f] > -1; }
					inline void getFaceIsBoundary(I f, bool * r) { *r = (a.faceBoundary[f] > -1); }
					inline I getFaceBoundaryID(I f) { return a.faceBoundary[f]; }
					inline T getFaceLambda(I f) { return a.faceLambda[f]; }
					inline T getFaceArea(I f) { return a.faceArea[f]; }
					inline cupcfd::geometry::euclidean::EuclideanVector3D<T> getFaceNorm(I f) {
						return cupcfd::geometry::euclidean::EuclideanVector3D<T>(a.faceNorm[3*f], a.faceNorm[3*f+1], a.faceNorm[3*f+2]);
					}
					inline void getFaceNorm(I f, cupcfd::geometry::euclidean::EuclideanVector3D<T>& n) {
						n.cmp[0] = a.faceNorm[3*f]; n.cmp[1] = a.faceNorm[3*f+1]; n.cmp[2] = a.faceNorm[3*f+2];
					}
					inline T getFaceRLencos(I f) { return a.faceRLencos[f]; }
					inline T getBoundaryDistance(I b) { return a.boundaryDistance[b]; }
					inline cupcfd::geometry::euclidean::EuclideanVector<T,3> getBoundaryShear(I b) {
						return cupcfd::geometry::euclidean::EuclideanVector<T,3>(a.boundaryShear[3*b], a.boundaryShear[3*b+1], a.boundaryShear[3*b+2]);
					}
					inline void setBoundaryShear(I b, cupcfd::geometry::euclidean::EuclideanVector<T,3>& v) {
						for (int d = 0; d < 3; d++) a.boundaryShear[3*b+d] = v.cmp[d];
					}
					inline cupcfd::geometry::euclidean::EuclideanVector<T,3> getRegionForceTangent(I r) {
						return cupcfd::geometry::euclidean::EuclideanVector<T,3>(a.regionForceTangent[3*r], a.regionForceTangent[3*r+1], a.regionForceTangent[3*r+2]);
					}
					inline void setRegionForceTangent(I r, cupcfd::geometry::euclidean::EuclideanVector<T,3>& v) {
						for (int d = 0; d < 3; d++) a.regionForceTangent[3*r+d] = v.cmp[d];
					}
					inline cupcfd::geometry::euclidean::EuclideanPoint<T,3> getFaceCenter(I f) {
						return cupcfd::geometry::euclidean::EuclideanPoint<T,3>(a.faceCenter[3*f], a.faceCenter[3*f+1], a.faceCenter[3*f+2]);
					}
					inline cupcfd::geometry::euclidean::EuclideanPoint<T,3> getFaceXpac(I f) {
						return cupcfd::geometry::euclidean::EuclideanPoint<T,3>(a.faceXpac[3*f], a.faceXpac[3*f+1], a.faceXpac[3*f+2]);
					}
					inline cupcfd::geometry::euclidean::EuclideanPoint<T,3> getFaceXnac(I f) {
						return cupcfd::geometry::euclidean::EuclideanPoint<T,3>(a.faceXnac[3*f], a.faceXnac[3*f+1], a.faceXnac[3*f+2]);
					}
					inline cupcfd::geometry::euclidean::EuclideanPoint<T,3> getCellCenter(I c) {
						return cupcfd::geometry::euclidean::EuclideanPoint<T,3>(a.cellCenter[3*c], a.cellCenter[3*c+1], a.cellCenter[3*c+2]);
					}
					inline void getCellVolume(I c, T * v) { *v = a.cellVolume[c]; }
					inline T getCellVolume(I c) { return a.cellVolume[c]; }
					inline I getBoundaryRegionID(I b) { return a.boundaryRegion[b]; }
					inline RType getRegionType(I r) { return (RType) a.regionType[r]; }
					inline T getRegionDen(I r) { return a.regionDen[r]; }
					inline I getBoundaryFaceID(I b) { return a.boundaryFace[b]; }
					inline T getRegionSplvl(I r) { return a.regionSplvl[r]; }
					inline cupcfd::geometry::euclidean::EuclideanVector<T,3> getRegionUVW(I r) {
						return cupcfd::geometry::euclidean::EuclideanVector<T,3>(a.regionUVW[3*r], a.regionUVW[3*r+1], a.regionUVW[3*r+2]);
					}
			};
		}
	}
}

#endif
