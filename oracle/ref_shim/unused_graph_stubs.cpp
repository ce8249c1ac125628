/*
 * Link-time stand-ins for the four DistributedAdjacencyList<int,int> members
 * that MeshSource<I,T,L>::buildDistributedAdjacencyList references
 * (src/geometry/mesh/interface/source/MeshSource.cpp). The oracle never calls
 * that method: it reads the generator's getters directly and lays the mesh
 * out the way a one-rank addData does. These definitions only let the
 * reference's generator link into oracle/_ref/libcupcfd_ref.so without the
 * MPI-dependent graph code. TEST INFRASTRUCTURE ONLY.
 */
#include "DistributedAdjacencyList.h"

namespace cupcfd { namespace data_structures {
template <> cupcfd::error::eCodes DistributedAdjacencyList<int,int>::addLocalNode(int) { return cupcfd::error::E_NOT_IMPLEMENTED; }
template <> cupcfd::error::eCodes DistributedAdjacencyList<int,int>::addUndirectedEdge(int, int) { return cupcfd::error::E_NOT_IMPLEMENTED; }
template <> void DistributedAdjacencyList<int,int>::reset() { }
template <> cupcfd::error::eCodes DistributedAdjacencyList<int,int>::finalize() { return cupcfd::error::E_NOT_IMPLEMENTED; }
} }
