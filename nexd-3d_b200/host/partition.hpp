// Domain decomposition of a descriptor into partitions with their halo
// descriptors: the data the reference's mesher hands each rank for
// nproc > 1 (METIS element partition, src/meshMod.f90:382-504; interface
// arrays mpi_neighbor / mpi_connection / mpi_ibool / mpi_ibt,
// src/meshMod.f90:669-1110).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/nexd.h"

namespace nexd {

struct PartData {
  nexd_desc desc{};
  nexd_halo_desc halo{};
  std::vector<double> metric, jac, fscale, nn, st, tt, rho, vpu, vsu, lam, mu, ylam, ymu, prof;
  std::vector<double> srcInt, srcang, srcM, stf, recInt;
  std::vector<int32_t> neighbor, face, ibn, pmlcheck, srcelem, srctype, srcbatch, recelem;
  std::vector<int32_t> peer, nface, helem, hside, peer_index, peer_node;
  std::vector<int32_t> elem_global, src_global, rec_global;  // 1-based ids in the whole mesh
};

// Element partition: `part` (K values, 0-based) when given, else recursive
// coordinate bisection of the centroids (3,K) into nparts parts whose sizes
// differ by at most one element.
std::vector<int32_t> bisect_partition(const double* centroid, int K, int nparts);

// Splits `d` by `part`.  Throws std::runtime_error on inconsistent input.
// The partitions share the operators (Dr, Ds, Dt, lift, invmass, fmask, wl)
// with `d`.
void split_descriptor(const nexd_desc& d, const std::vector<int32_t>& part, int nparts, std::vector<PartData>& out);

}  // namespace nexd
