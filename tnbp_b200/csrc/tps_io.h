// Checkpoint files of the PEPS state (SaveTPS / LoadTPS); see tps_io.cpp.
#pragma once
#include <complex>
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "host_setup.h"

namespace tnbp_host {

struct TpsTensor {
  std::vector<int32_t> shape;
  std::vector<std::complex<double>> data;  // column-major
};

// One rank's part of the state, in the field order of SaveTPS.
struct TpsState {
  std::vector<TpsTensor> V;                   // site tensors, SiteIdx order
  std::vector<int32_t> site_idx;              // site labels
  std::vector<std::pair<int32_t, int32_t>> site_rank;  // Site_To_MpiRank
  std::vector<TpsTensor> E;                   // 2 |EdgeIdx| messages
  std::vector<int32_t> edge_idx;              // edge ids
};

void tps_write(const std::string& path, const TpsState& st);
TpsState tps_read(const std::string& path);

// The whole state of one edge list, held by a single rank, from packed
// arrays: site tensors in sorted-site order, each of shape (bond dims in leg
// order..., phys), then the 2|E| messages, message m of shape
// (bond_dim[m % ne], bond_dim[m % ne]).
TpsState tps_whole(const Edges& edges, const std::vector<int>& bond_dim, const std::vector<int>& phys_dim,
                   const std::complex<double>* site_data, const std::complex<double>* msg_data);

// Checks that st holds the whole state of `edges` on one rank and returns the
// bond and physical dimensions it implies.
void tps_check_whole(const TpsState& st, const Edges& edges, std::vector<int>& bond_dim,
                     std::vector<int>& phys_dim);

}  // namespace tnbp_host
