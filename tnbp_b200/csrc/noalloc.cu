// One directed BP message computed without any device allocation.
//
// Same arithmetic as one message of the sweep (bp.h:128-175): the site
// tensor absorbs the incoming messages on every leg but the target
// (k_leg_apply, one launch per leg), the result is contracted with conj(V)
// over all legs but the target (k_gram, split-K partials) and the sum is
// normalized (k_msg_finalize).  The intermediate tensors, the Gram partials
// and the task descriptors live in g_noalloc_scratch, a file-scope
// __device__ array, instead of memory from cudaMalloc/cudaMallocAsync.
//
// Who needs this: code that runs inside a host framework which owns the
// whole device-memory budget (a pre-reserved arena, an allocator that must
// account for every byte, a co-tenant of the served loop) and may not call
// cudaMalloc, and code on a stream-ordered pipeline where cudaMalloc's
// implicit device synchronization is not acceptable.  Such callers pass
// device pointers to the inputs and the output and get no allocation.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tnbp_b200.h"
#include "engine.h"
#include "kernels.cuh"

namespace tnbp {
namespace {

constexpr size_t kTaskBytes = size_t(64) << 10;
constexpr size_t kPartialBytes = size_t(4) << 20;
constexpr size_t kBufElems = size_t(TNBP_NOALLOC_MAX_SITE_ELEMS);
constexpr size_t kScratchBytes = kTaskBytes + kPartialBytes + 2 * kBufElems * sizeof(double2);

// Shared by every call on a device; held by every GPU that loads the library
// until the process exits (about 36 MiB).
__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device.  The name of a
// __device__ variable is only a host-side stand-in: the address must come
// from cudaGetSymbolAddress, once per device, with that device current.
unsigned char* scratch_for_current_device() {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) throw Error(TNBP_EINVAL, "device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      throw Error(TNBP_ECUDA, std::string("cudaGetSymbolAddress(g_noalloc_scratch) failed: ") +
                                  cudaGetErrorString(e));
    }
    g_scratch_ptr[dev] = p;
  }
  return static_cast<unsigned char*>(g_scratch_ptr[dev]);
}

// Every descriptor of one call, stored at the start of the scratch array.
struct NoallocTasks {
  long long zero;  // the one-entry block-prefix array of every launch
  int nleg;
  LegTask leg[kMaxLegs];
  GramTask gram;
  MsgTask msg;
};

// Copies the by-value parameter block into device memory (word by word).
__global__ void k_store_noalloc_tasks(const NoallocTasks pack, NoallocTasks* dst) {
  static_assert(sizeof(NoallocTasks) % sizeof(unsigned int) == 0, "word copy");
  const unsigned int* src = reinterpret_cast<const unsigned int*>(&pack);
  unsigned int* out = reinterpret_cast<unsigned int*>(dst);
  for (size_t i = threadIdx.x; i < sizeof(NoallocTasks) / sizeof(unsigned int); i += blockDim.x) out[i] = src[i];
}

void message_noalloc(const double* site, const int32_t* shape, int32_t rank, int32_t target,
                     const double* const* msgs, double* out, cudaStream_t stream) {
  if (!site || !shape || !msgs || !out) throw Error(TNBP_EINVAL, "NULL argument");
  const int g = rank - 1;
  if (g < 1 || g > kMaxLegs) throw Error(TNBP_EINVAL, "rank must be 2.." + std::to_string(kMaxLegs + 1));
  if (target < 0 || target >= g) throw Error(TNBP_EINVAL, "target leg out of range");
  size_t n = 1;
  for (int k = 0; k < rank; ++k) {
    if (shape[k] < 1) throw Error(TNBP_EINVAL, "dimensions must be >= 1");
    if (k < g && shape[k] > 128) throw Error(TNBP_EINVAL, "bond dimension above 128");
    n *= (size_t)shape[k];
  }
  if (n > kBufElems)
    throw Error(TNBP_EINVAL, "site tensor of " + std::to_string(n) + " elements exceeds the no-allocation limit of " +
                                 std::to_string(kBufElems) + " complex128 elements");
  for (int k = 0; k < g; ++k)
    if (k != target && !msgs[k]) throw Error(TNBP_EINVAL, "incoming message pointer is NULL");

  unsigned char* base = scratch_for_current_device();
  unsigned char* tasks_area = base;
  double2* partial = reinterpret_cast<double2*>(base + kTaskBytes);
  double2* buf[2] = {reinterpret_cast<double2*>(base + kTaskBytes + kPartialBytes),
                     reinterpret_cast<double2*>(base + kTaskBytes + kPartialBytes) + kBufElems};

  // leg contractions: every leg but the target, in order
  std::vector<LegTask> legs;
  const void* src = site;
  int which = 0;
  for (int k = 0; k < g; ++k) {
    if (k == target) continue;
    long long L = 1, R = 1;
    for (int q = 0; q < k; ++q) L *= shape[q];
    for (int q = k + 1; q < rank; ++q) R *= shape[q];
    LegTask t;
    t.in = src;
    t.out = buf[which];
    t.mat = msgs[k];
    t.L = L; t.R = R; t.Din = shape[k]; t.Dout = shape[k];
    set_leg_divisors(t);
    t.block_begin = 0;
    legs.push_back(t);
    src = buf[which];
    which ^= 1;
  }
  // Gram over all legs but the target
  GramTask gt;
  gt.A = src;
  gt.B = site;
  long long L = 1, M = 1;
  for (int q = 0; q < target; ++q) L *= shape[q];
  for (int q = target + 1; q < rank; ++q) M *= shape[q];
  gt.L = L; gt.M = M; gt.D = shape[target]; gt.P = 1; gt.C = shape[target];
  gt.ctiles = (gt.C + kColTile - 1) / kColTile;
  gt.Q = L * M;
  long long cr = ((gt.Q / 16) + kRowTile - 1) / kRowTile * kRowTile;
  gt.chunk_rows = std::max<long long>(256, std::min<long long>(4096, cr));
  gt.nchunk = (int)((gt.Q + gt.chunk_rows - 1) / gt.chunk_rows);
  if ((size_t)gt.nchunk * gt.C * gt.C * sizeof(double2) > kPartialBytes)
    throw Error(TNBP_EINVAL, "Gram partials exceed the no-allocation partial area");
  gt.partial = partial;
  gt.block_begin = 0;
  MsgTask mt;
  mt.partial = partial;
  mt.nchunk = gt.nchunk;
  mt.C = gt.C;
  mt.out = out;
  mt.old = nullptr;
  mt.dist = nullptr;
  mt.norm_out = nullptr;

  // Task descriptors: passed BY VALUE as the parameter block of one small
  // kernel that stores them into the scratch array, so nothing is read from
  // host memory after this call returns (a pageable host copy would not be
  // stream-ordered like the kernels that read the descriptors).
  NoallocTasks pack{};
  pack.nleg = (int)legs.size();
  for (size_t i = 0; i < legs.size(); ++i) pack.leg[i] = legs[i];
  pack.gram = gt;
  pack.msg = mt;
  NoallocTasks* d_pack = reinterpret_cast<NoallocTasks*>(tasks_area);
  static_assert(sizeof(NoallocTasks) <= kTaskBytes, "task area too small");
  k_store_noalloc_tasks<<<1, 128, 0, stream>>>(pack, d_pack);
  CK(cudaGetLastError());
  note_launch(1);
  const long long* d_zero = &d_pack->zero;
  const GramTask* d_gram = &d_pack->gram;
  const MsgTask* d_msg = &d_pack->msg;

  prepare_kernels(TNBP_C128);
  for (size_t i = 0; i < legs.size(); ++i) {
    const LegTask& t = legs[i];
    const long long nb = (t.L * t.R + kRowTile - 1) / kRowTile;
    const size_t smem = (size_t)(kRowTile * (t.Din + 1) + t.Din * (kColTile + 1)) * sizeof(double2);
    k_leg_apply<double><<<(unsigned)nb, kThreads, smem, stream>>>(&d_pack->leg[i], d_zero, 1, t.Din);
    CK(cudaGetLastError());
    note_launch(1);
  }
  k_gram<double><<<(unsigned)((long long)gt.nchunk * gt.ctiles * gt.ctiles), kThreads, 0, stream>>>(d_gram, d_zero, 1);
  CK(cudaGetLastError());
  k_msg_finalize<double><<<1, kThreads, 0, stream>>>(d_msg);
  CK(cudaGetLastError());
  note_launch(2);
}

}  // namespace
}  // namespace tnbp

extern "C" int tnbp_bp_message_noalloc(const double* site, const int32_t* shape, int32_t rank, int32_t target,
                                       const double* const* msgs_in, double* msg_out, void* stream) {
  try {
    tnbp::g_last_error.clear();
    tnbp::message_noalloc(site, shape, rank, target, msgs_in, msg_out, static_cast<cudaStream_t>(stream));
    return TNBP_OK;
  } catch (const tnbp::Error& e) {
    tnbp::g_last_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    tnbp::g_last_error = e.what();
    return TNBP_EINVAL;
  }
}
