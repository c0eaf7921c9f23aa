// Checkpoint files of the PEPS state in the layout of SaveTPS / LoadTPS
// (include/tnbp/ptns/function/iotps.h:37-105), little-endian:
//   size_t |V|, size_t |Site_To_MpiRank|, size_t |EdgeIdx|
//   |V| tensor records (site tensors)
//   |V| int32 SiteIdx
//   |Site_To_MpiRank| pairs of int32 (site label, rank), in key order
//   2 |EdgeIdx| tensor records (messages; m < |EdgeIdx| computed at the
//   edge's first site, the rest at its second)
//   |EdgeIdx| int32 EdgeIdx
// A tensor record is what tci::save writes through the tensor's
// StreamWrite (external/min-tci/include/tci/gqten/io.h:40-63).  gqten
// itself is not available, so its record layout is the one restated for
// gqten::tensor<std::complex<double>> with this project's CPU stand-in:
//   uint64 order, int32 shape[order], complex128 scale (1 for a tensor of
//   order >= 1), complex128 data[prod(shape)] column-major.
// Elements are always complex128 (the reference's complex<double> apps).
#include "tps_io.h"

#include <algorithm>
#include <fstream>
#include <numeric>

namespace tnbp_host {

namespace {

constexpr int kBadFile = -1;  // TNBP_EINVAL

template <class T>
void put(std::ofstream& f, const T& v) {
  f.write(reinterpret_cast<const char*>(&v), sizeof(T));
}

void put_tensor(std::ofstream& f, const TpsTensor& t) {
  const uint64_t order = t.shape.size();
  put(f, order);
  f.write(reinterpret_cast<const char*>(t.shape.data()), sizeof(int32_t) * order);
  put(f, std::complex<double>(1.0, 0.0));
  f.write(reinterpret_cast<const char*>(t.data.data()), sizeof(std::complex<double>) * t.data.size());
}

struct Reader {
  std::ifstream f;
  std::string path;
  template <class T>
  T get() {
    T v{};
    f.read(reinterpret_cast<char*>(&v), sizeof(T));
    if (!f) throw HostError(kBadFile, "checkpoint " + path + ": unexpected end of file");
    return v;
  }
  TpsTensor tensor() {
    TpsTensor t;
    const uint64_t order = get<uint64_t>();
    if (order == 0 || order > 64) throw HostError(kBadFile, "checkpoint " + path + ": bad tensor order");
    t.shape.resize(order);
    uint64_t n = 1;
    for (auto& d : t.shape) {
      d = get<int32_t>();
      if (d < 1 || d > (1 << 20)) throw HostError(kBadFile, "checkpoint " + path + ": bad tensor shape");
      n *= (uint64_t)d;
      if (n > (uint64_t(1) << 36)) throw HostError(kBadFile, "checkpoint " + path + ": tensor too large");
    }
    // the record's scale multiplies every stored element (1 in files the
    // reference writes for tensors of order >= 1)
    const std::complex<double> scale = get<std::complex<double>>();
    if (!std::isfinite(scale.real()) || !std::isfinite(scale.imag()))
      throw HostError(kBadFile, "checkpoint " + path + ": non-finite tensor scale");
    t.data.resize(n);
    f.read(reinterpret_cast<char*>(t.data.data()), (std::streamsize)(sizeof(std::complex<double>) * n));
    if (!f) throw HostError(kBadFile, "checkpoint " + path + ": unexpected end of file");
    if (scale != std::complex<double>(1.0, 0.0))
      for (auto& x : t.data) x *= scale;
    return t;
  }
};

}  // namespace

void tps_write(const std::string& path, const TpsState& st) {
  std::ofstream f(path, std::ios::binary | std::ios::trunc);
  if (!f) throw HostError(kBadFile, "cannot open " + path + " for writing");
  put(f, (uint64_t)st.V.size());
  put(f, (uint64_t)st.site_rank.size());
  put(f, (uint64_t)st.edge_idx.size());
  for (const auto& t : st.V) put_tensor(f, t);
  for (int32_t s : st.site_idx) put(f, s);
  for (const auto& kv : st.site_rank) { put(f, kv.first); put(f, kv.second); }
  for (const auto& t : st.E) put_tensor(f, t);
  for (int32_t m : st.edge_idx) put(f, m);
  f.flush();
  if (!f) throw HostError(kBadFile, "write to " + path + " failed");
}

TpsState tps_read(const std::string& path) {
  Reader r;
  r.path = path;
  r.f.open(path, std::ios::binary);
  if (!r.f) throw HostError(kBadFile, "cannot open " + path);
  const uint64_t nV = r.get<uint64_t>(), nM = r.get<uint64_t>(), nE = r.get<uint64_t>();
  if (nV > (1u << 24) || nM > (1u << 24) || nE > (1u << 24))
    throw HostError(kBadFile, "checkpoint " + path + ": implausible header");
  TpsState st;
  st.V.reserve(nV);
  for (uint64_t i = 0; i < nV; ++i) st.V.push_back(r.tensor());
  for (uint64_t i = 0; i < nV; ++i) st.site_idx.push_back(r.get<int32_t>());
  for (uint64_t i = 0; i < nM; ++i) {
    const int32_t k = r.get<int32_t>();
    st.site_rank.push_back({k, r.get<int32_t>()});
  }
  st.E.reserve(2 * nE);
  for (uint64_t i = 0; i < 2 * nE; ++i) st.E.push_back(r.tensor());
  for (uint64_t i = 0; i < nE; ++i) st.edge_idx.push_back(r.get<int32_t>());
  return st;
}

TpsState tps_whole(const Edges& edges, const std::vector<int>& bond_dim, const std::vector<int>& phys_dim,
                   const std::complex<double>* site_data, const std::complex<double>* msg_data) {
  const auto sites = site_labels(edges);
  const size_t ns = sites.size(), ne = edges.size();
  if (bond_dim.size() != ne || phys_dim.size() != ns) throw HostError(kBadFile, "dimension lists do not match");
  TpsState st;
  size_t o = 0;
  for (size_t s = 0; s < ns; ++s) {
    TpsTensor t;
    for (int m : surrounding_bonds(edges, sites[s])) t.shape.push_back(bond_dim[m]);
    t.shape.push_back(phys_dim[s]);
    size_t n = 1;
    for (int d : t.shape) n *= (size_t)d;
    t.data.assign(site_data + o, site_data + o + n);
    o += n;
    st.V.push_back(std::move(t));
    st.site_idx.push_back(sites[s]);
    st.site_rank.push_back({sites[s], 0});
  }
  o = 0;
  for (size_t m = 0; m < 2 * ne; ++m) {
    const int D = bond_dim[m % ne];
    TpsTensor t;
    t.shape = {D, D};
    t.data.assign(msg_data + o, msg_data + o + (size_t)D * D);
    o += (size_t)D * D;
    st.E.push_back(std::move(t));
  }
  for (size_t m = 0; m < ne; ++m) st.edge_idx.push_back((int32_t)m);
  return st;
}

void tps_check_whole(const TpsState& st, const Edges& edges, std::vector<int>& bond_dim,
                     std::vector<int>& phys_dim) {
  const auto sites = site_labels(edges);
  const size_t ns = sites.size(), ne = edges.size();
  if (st.V.size() != ns || st.edge_idx.size() != ne)
    throw HostError(kBadFile, "checkpoint holds " + std::to_string(st.V.size()) + " sites and " +
                                  std::to_string(st.edge_idx.size()) + " edges, the edge list " +
                                  std::to_string(ns) + " and " + std::to_string(ne) +
                                  " (a checkpoint of one rank of several?)");
  for (size_t s = 0; s < ns; ++s)
    if (st.site_idx[s] != sites[s]) throw HostError(kBadFile, "checkpoint site labels differ from the edge list's");
  for (size_t m = 0; m < ne; ++m)
    if (st.edge_idx[m] != (int32_t)m) throw HostError(kBadFile, "checkpoint edge ids are not 0 .. |E|-1");
  if (st.site_rank.size() != ns) throw HostError(kBadFile, "checkpoint site-to-rank map is partial");
  bond_dim.assign(ne, 0);
  phys_dim.assign(ns, 0);
  for (size_t s = 0; s < ns; ++s) {
    const auto legs = surrounding_bonds(edges, sites[s]);
    const auto& sh = st.V[s].shape;
    if (sh.size() != legs.size() + 1) throw HostError(kBadFile, "checkpoint site tensor order != degree + 1");
    for (size_t k = 0; k < legs.size(); ++k) {
      int& d = bond_dim[legs[k]];
      if (d != 0 && d != sh[k]) throw HostError(kBadFile, "checkpoint site tensors disagree on a bond dimension");
      d = sh[k];
    }
    phys_dim[s] = sh.back();
  }
  for (size_t m = 0; m < 2 * ne; ++m) {
    const auto& sh = st.E[m].shape;
    const int D = bond_dim[m % ne];
    if (sh.size() != 2 || sh[0] != D || sh[1] != D)
      throw HostError(kBadFile, "checkpoint message shape does not match its bond dimension");
  }
}

}  // namespace tnbp_host
