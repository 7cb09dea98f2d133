// Domain decomposition of a descriptor (see partition.hpp).
#include "partition.hpp"

#include <algorithm>
#include <numeric>
#include <stdexcept>
#include <string>

namespace nexd {

namespace {

// Splits elems[lo, hi) into nparts parts along the axis of largest centroid
// extent, the first floor(nparts/2) parts taking their share of the elements.
void bisect(const double* c, std::vector<int>& elems, size_t lo, size_t hi, int nparts, int first,
            std::vector<int32_t>& part) {
  if (nparts == 1) {
    for (size_t i = lo; i < hi; ++i) part[elems[i]] = first;
    return;
  }
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (size_t i = lo; i < hi; ++i)
    for (int k = 0; k < 3; ++k) {
      mn[k] = std::min(mn[k], c[3 * size_t(elems[i]) + k]);
      mx[k] = std::max(mx[k], c[3 * size_t(elems[i]) + k]);
    }
  int ax = 0;
  for (int k = 1; k < 3; ++k)
    if (mx[k] - mn[k] > mx[ax] - mn[ax]) ax = k;
  const int left = nparts / 2;
  const size_t n = hi - lo, nl = (n * size_t(left) + size_t(nparts) / 2) / size_t(nparts);
  // ties broken by element id, so the split does not depend on the sort
  auto less = [&](int a, int b) {
    const double ca = c[3 * size_t(a) + ax], cb = c[3 * size_t(b) + ax];
    return ca < cb || (ca == cb && a < b);
  };
  std::nth_element(elems.begin() + lo, elems.begin() + lo + nl, elems.begin() + hi, less);
  bisect(c, elems, lo, lo + nl, left, first, part);
  bisect(c, elems, lo + nl, hi, nparts - left, first + left, part);
}

template <class T>
void take(const T* src, int stride, const std::vector<int>& list, std::vector<T>& dst) {
  dst.clear();
  if (!src) return;
  dst.reserve(list.size() * size_t(stride));
  for (int e : list) dst.insert(dst.end(), src + size_t(e) * stride, src + size_t(e + 1) * stride);
}

}  // namespace

std::vector<int32_t> bisect_partition(const double* centroid, int K, int nparts) {
  if (!centroid) throw std::runtime_error("partition: centroids needed when no element partition is given");
  if (nparts < 1 || nparts > K) throw std::runtime_error("partition: part count out of 1..K");
  std::vector<int> elems(K);
  std::iota(elems.begin(), elems.end(), 0);
  std::vector<int32_t> part(K, 0);
  bisect(centroid, elems, 0, size_t(K), nparts, 0, part);
  return part;
}

void split_descriptor(const nexd_desc& d, const std::vector<int32_t>& part, int nparts, std::vector<PartData>& out) {
  const int K = d.nelem, Np = d.Np, NpF = d.NpF, nMB = d.attenuation ? d.nMB : 0;
  if (K <= 0 || int(part.size()) != K) throw std::runtime_error("partition: element count mismatch");
  if (nparts < 1 || nparts > K) throw std::runtime_error("partition: part count out of 1..K");
  for (int k = 0; k < 4 * K; ++k)
    if (d.neighbor[k] == 0 && d.face[k] == NEXD_FACE_PARTITION)
      throw std::runtime_error("partition: the descriptor is a partition already");
  std::vector<std::vector<int>> elems(nparts);
  for (int e = 0; e < K; ++e) {
    if (part[e] < 0 || part[e] >= nparts) throw std::runtime_error("partition: element partition out of 0..nparts-1");
    elems[part[e]].push_back(e);
  }
  for (int p = 0; p < nparts; ++p)
    if (elems[p].empty()) throw std::runtime_error("partition: an empty partition");
  std::vector<int> local(K);
  for (int p = 0; p < nparts; ++p)
    for (size_t i = 0; i < elems[p].size(); ++i) local[elems[p][i]] = int(i);

  // shared faces of each partition, grouped by neighbour partition in
  // connection order (element, then side), and each face's index in its group
  std::vector<std::vector<std::vector<int>>> groups(nparts, std::vector<std::vector<int>>(nparts));
  std::vector<int> gindex(size_t(4) * K, -1);
  for (int p = 0; p < nparts; ++p)
    for (int e : elems[p])
      for (int f = 0; f < 4; ++f) {
        const int nb = d.neighbor[4 * e + f];
        if (nb <= 0 || part[nb - 1] == p) continue;
        auto& g = groups[p][part[nb - 1]];
        gindex[4 * e + f] = int(g.size());
        g.push_back(4 * e + f);
      }

  out.assign(nparts, PartData{});
  for (int p = 0; p < nparts; ++p) {
    PartData& o = out[p];
    const std::vector<int>& L = elems[p];
    const int Kp = int(L.size());
    take(d.metric, 9, L, o.metric);
    take(d.jacobian, 1, L, o.jac);
    take(d.fscale, 4, L, o.fscale);
    take(d.nnormal, 12, L, o.nn);
    take(d.stangential, 12, L, o.st);
    take(d.ttangential, 12, L, o.tt);
    take(d.rho, 1, L, o.rho);
    take(d.vpu, 1, L, o.vpu);
    take(d.vsu, 1, L, o.vsu);
    take(d.lambdau, 1, L, o.lam);
    take(d.muu, 1, L, o.mu);
    if (nMB > 0) {
      take(d.ylambda, nMB, L, o.ylam);
      take(d.ymu, nMB, L, o.ymu);
    }
    if (d.set_pml) {
      take(d.pmlcheck, 1, L, o.pmlcheck);
      o.prof.resize(size_t(Kp) * Np * 9);
      for (int c = 0; c < 9; ++c)
        for (int i = 0; i < Kp; ++i)
          std::copy(d.pml_profiles + size_t(c) * K * Np + size_t(L[i]) * Np,
                    d.pml_profiles + size_t(c) * K * Np + size_t(L[i] + 1) * Np,
                    o.prof.begin() + size_t(c) * Kp * Np + size_t(i) * Np);
    }
    // connectivity in local numbering; shared faces coded -3
    o.neighbor.assign(size_t(4) * Kp, 0);
    o.face.assign(size_t(4) * Kp, 0);
    o.ibn.assign(size_t(4) * Kp * NpF, 0);
    for (int i = 0; i < Kp; ++i) {
      const int e = L[i];
      for (int f = 0; f < 4; ++f) {
        const int nb = d.neighbor[4 * e + f];
        const size_t k = size_t(4) * i + f;
        if (nb == 0) {
          o.face[k] = d.face[4 * e + f];
        } else if (part[nb - 1] != p) {
          o.face[k] = NEXD_FACE_PARTITION;
        } else {
          o.neighbor[k] = local[nb - 1] + 1;
          o.face[k] = d.face[4 * e + f];
          for (int j = 0; j < NpF; ++j) {
            const long long m = (long long)d.ibn[(size_t(e) * 4 + f) * NpF + j] - 1 - (long long)(nb - 1) * Np;
            if (m < 0 || m >= Np) throw std::runtime_error("partition: ibn does not point into the neighbour element");
            o.ibn[k * NpF + j] = int32_t((long long)local[nb - 1] * Np + m + 1);
          }
        }
      }
    }
    // halo: neighbours in ascending partition order
    for (int q = 0; q < nparts; ++q) {
      const auto& g = groups[p][q];
      if (g.empty()) continue;
      o.peer.push_back(q + 1);
      o.nface.push_back(int32_t(g.size()));
      for (int key : g) {
        const int e = key / 4, f = key % 4;
        const int nb = d.neighbor[key], fn = d.face[key] - 1;
        if (fn < 0 || fn > 3) throw std::runtime_error("partition: interior face without neighbour face id");
        const int ri = gindex[4 * (nb - 1) + fn];
        if (ri < 0 || d.neighbor[4 * (nb - 1) + fn] != e + 1)
          throw std::runtime_error("partition: neighbour face does not point back");
        o.helem.push_back(local[e] + 1);
        o.hside.push_back(f + 1);
        o.peer_index.push_back(ri + 1);
        for (int j = 0; j < NpF; ++j) {
          const long long m = (long long)d.ibn[(size_t(e) * 4 + f) * NpF + j] - 1 - (long long)(nb - 1) * Np;
          int pos = -1;
          for (int jj = 0; jj < NpF; ++jj)
            if (d.fmask[fn * NpF + jj] - 1 == m) pos = jj;
          if (pos < 0) throw std::runtime_error("partition: matching node not on the neighbour's face");
          o.peer_node.push_back(pos + 1);
        }
      }
    }
    // sources and receivers inside the partition, in their original order
    for (int s = 0; s < d.nsrc; ++s) {
      const int e = d.srcelem[s] - 1;
      if (e < 0 || e >= K) throw std::runtime_error("partition: srcelem out of range");
      if (part[e] != p) continue;
      o.src_global.push_back(s + 1);
      o.srcelem.push_back(local[e] + 1);
      o.srctype.push_back(d.srctype[s]);
      if (d.srcbatch) o.srcbatch.push_back(d.srcbatch[s]);
      o.srcInt.insert(o.srcInt.end(), d.srcInt + size_t(s) * Np, d.srcInt + size_t(s + 1) * Np);
      if (d.srcangle_force) o.srcang.insert(o.srcang.end(), d.srcangle_force + 3 * s, d.srcangle_force + 3 * s + 3);
      if (d.srcM) o.srcM.insert(o.srcM.end(), d.srcM + 6 * s, d.srcM + 6 * s + 6);
      const size_t ns = size_t(d.stf_per_step) * d.nt;
      o.stf.insert(o.stf.end(), d.stf + ns * s, d.stf + ns * (s + 1));
    }
    for (int r = 0; r < d.nrec; ++r) {
      const int e = d.recelem[r] - 1;
      if (e < 0 || e >= K) throw std::runtime_error("partition: recelem out of range");
      if (part[e] != p) continue;
      o.rec_global.push_back(r + 1);
      o.recelem.push_back(local[e] + 1);
      o.recInt.insert(o.recInt.end(), d.recInt + size_t(r) * Np, d.recInt + size_t(r + 1) * Np);
    }
    for (int e : L) o.elem_global.push_back(e + 1);

    nexd_desc& pd = o.desc;
    pd = d;  // scalars and the shared operators
    pd.nelem = Kp;
    pd.metric = o.metric.data();
    pd.jacobian = o.jac.data();
    pd.fscale = o.fscale.data();
    pd.nnormal = o.nn.data();
    pd.stangential = o.st.data();
    pd.ttangential = o.tt.data();
    pd.rho = o.rho.data();
    pd.vpu = o.vpu.data();
    pd.vsu = o.vsu.data();
    pd.lambdau = o.lam.data();
    pd.muu = o.mu.data();
    pd.ylambda = nMB > 0 ? o.ylam.data() : d.ylambda;
    pd.ymu = nMB > 0 ? o.ymu.data() : d.ymu;
    pd.neighbor = o.neighbor.data();
    pd.face = o.face.data();
    pd.ibn = o.ibn.data();
    pd.pmlcheck = d.set_pml ? o.pmlcheck.data() : d.pmlcheck;
    pd.pml_profiles = d.set_pml ? o.prof.data() : d.pml_profiles;
    pd.nsrc = int32_t(o.srcelem.size());
    pd.srcelem = o.srcelem.data();
    pd.srctype = o.srctype.data();
    pd.srcInt = o.srcInt.data();
    pd.srcangle_force = d.srcangle_force ? o.srcang.data() : nullptr;
    pd.srcM = d.srcM ? o.srcM.data() : nullptr;
    pd.stf = o.stf.data();
    pd.srcbatch = d.srcbatch ? o.srcbatch.data() : nullptr;
    pd.nrec = int32_t(o.recelem.size());
    pd.recelem = o.recelem.data();
    pd.recInt = o.recInt.data();

    nexd_halo_desc& h = o.halo;
    h.partition = p + 1;
    h.npeer = int32_t(o.peer.size());
    h.peer = o.peer.data();
    h.nface = o.nface.data();
    h.elem = o.helem.data();
    h.side = o.hside.data();
    h.peer_index = o.peer_index.data();
    h.peer_node = o.peer_node.data();
  }
}

}  // namespace nexd
