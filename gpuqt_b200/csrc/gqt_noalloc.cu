// gqt_chebyshev_step_noalloc: the fused Chebyshev step + moment of the FP64 form
// with its reduction scratch in a static device array, for callers that cannot let
// the library call cudaMalloc (see include/gpuqt.h). No host or device allocation
// happens on any path of this file after the per-device set-up below, which itself
// only looks up an address.
#include <mutex>

#include "gqt_internal.h"
#include "gqt_kernels.cuh"

namespace {

using gqt::Dot;
using gqt::ExactArith;
using gqt::kApply;
using gqt::kBlock;
using gqt::kCheb;
using gqt::Op;

// Block partials of the moment sums (32 bytes per block and vector), then the
// arrival counter of the last-block reduction on its own 256-byte line.
constexpr size_t kPartialBytes = GQT_NOALLOC_SCRATCH_BYTES;
constexpr size_t kScratchBytes = kPartialBytes + 256;
static __device__ __align__(256) unsigned char g_step_scratch[kScratchBytes];

// Per-device set-up, kept in fixed tables so that no call allocates.
constexpr int kMaxDevices = 64;
// V in {1, 4, 16} x Z in {3, 4, 6, any} x mode x operator format (ELL arrays, coded)
constexpr int kKernels = 3 * 4 * 2 * 2;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices];
int g_sms[kMaxDevices];
int g_blocks_per_sm[kMaxDevices][kKernels];

int v_index(int nvec) { return nvec == 1 ? 0 : nvec == 4 ? 1 : 2; }

int z_index(int z) { return z == 3 ? 0 : z == 4 ? 1 : z == 6 ? 2 : 3; }

template <int V, int Z, int MODE, bool C>
const void* kernel_of()
{
  return (const void*)gqt::k_step<double2, V, Z, ExactArith, MODE, true, C>;
}

template <int V, int MODE, bool C>
const void* kernel_for_z(int z)
{
  switch (z_index(z)) {
    case 0:
      return kernel_of<V, 3, MODE, C>();
    case 1:
      return kernel_of<V, 4, MODE, C>();
    case 2:
      return kernel_of<V, 6, MODE, C>();
    default:
      return kernel_of<V, 0, MODE, C>();
  }
}

template <bool C>
const void* kernel_for_c(int nvec, int z, int mode)
{
  switch (v_index(nvec)) {
    case 0:
      return mode == 0 ? kernel_for_z<1, kApply, C>(z) : kernel_for_z<1, kCheb, C>(z);
    case 1:
      return mode == 0 ? kernel_for_z<4, kApply, C>(z) : kernel_for_z<4, kCheb, C>(z);
    default:
      return mode == 0 ? kernel_for_z<16, kApply, C>(z) : kernel_for_z<16, kCheb, C>(z);
  }
}

const void* kernel_for(int nvec, int z, int mode, bool coded)
{
  return coded ? kernel_for_c<true>(nvec, z, mode) : kernel_for_c<false>(nvec, z, mode);
}

// Once per device, with that device current: the array's device address (host code
// sees only a host-side stand-in under its name) and the launch limits. A coded
// kernel's limit is taken with the largest operator table in shared memory, so the
// grid never exceeds the blocks that are resident at once.
gqt_status setup(int dev, int nvec, int z, int mode, bool coded, int* blocks_per_sm)
{
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_step_scratch);
    if (e != cudaSuccess)
      return gqt::cuda_fail(e, "cudaGetSymbolAddress(g_step_scratch)", __FILE__, __LINE__);
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
      return gqt::cuda_fail(e, "cudaDeviceGetAttribute", __FILE__, __LINE__);
    g_sms[dev] = sms > 0 ? sms : 1;
    g_scratch_addr[dev] = p;
  }
  const int k = ((v_index(nvec) * 4 + z_index(z)) * 2 + mode) * 2 + (coded ? 1 : 0);
  if (g_blocks_per_sm[dev][k] == 0) {
    int b = 0;
    const size_t smem = coded ? (size_t)GQT_MAX_CODES * 28 : 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &b, kernel_for(nvec, z, mode, coded), kBlock, smem);
    if (e != cudaSuccess)
      return gqt::cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor", __FILE__,
                            __LINE__);
    g_blocks_per_sm[dev][k] = b > 0 ? b : 1;
  }
  *blocks_per_sm = g_blocks_per_sm[dev][k];
  return GQT_OK;
}

template <int V, int MODE, bool C>
void launch_c(int grid, cudaStream_t s, const Op& op, const double2* t0, const double2* t1,
              double2* out, const double2* left, const Dot& d)
{
  const size_t smem = gqt::op_smem_bytes(op);  // the coded table; 0 on the ELL arrays
  switch (z_index(op.z)) {
    case 0:
      gqt::k_step<double2, V, 3, ExactArith, MODE, true, C><<<grid, kBlock, smem, s>>>(
        op, t0, t1, out, left, d);
      break;
    case 1:
      gqt::k_step<double2, V, 4, ExactArith, MODE, true, C><<<grid, kBlock, smem, s>>>(
        op, t0, t1, out, left, d);
      break;
    case 2:
      gqt::k_step<double2, V, 6, ExactArith, MODE, true, C><<<grid, kBlock, smem, s>>>(
        op, t0, t1, out, left, d);
      break;
    default:
      gqt::k_step<double2, V, 0, ExactArith, MODE, true, C><<<grid, kBlock, smem, s>>>(
        op, t0, t1, out, left, d);
      break;
  }
}

template <int V, int MODE>
void launch(int grid, cudaStream_t s, const Op& op, const double2* t0, const double2* t1,
            double2* out, const double2* left, const Dot& d)
{
  if (op.code)
    launch_c<V, MODE, true>(grid, s, op, t0, t1, out, left, d);
  else
    launch_c<V, MODE, false>(grid, s, op, t0, t1, out, left, d);
}

}  // namespace

extern "C" gqt_status gqt_chebyshev_step_noalloc(const gqt_ham* h, int mode, const gqt_vec* t0,
                                                 const gqt_vec* t1, gqt_vec* out,
                                                 const gqt_vec* left, void* mu_dev)
{
  const char* w = "gqt_chebyshev_step_noalloc";
  if (!h || !t1 || !out || !left || !mu_dev || (mode == 1 && !t0))
    return gqt::fail(GQT_ERR_ARG, "%s: null argument", w);
  if (mode != 0 && mode != 1)
    return gqt::fail(GQT_ERR_ARG, "%s: mode must be 0 (first step) or 1 (got %d)", w, mode);
  const gqt_vec* vs[4] = {t1, out, left, mode == 1 ? t0 : t1};
  for (const gqt_vec* v : vs) {
    if (!v->data || v->n != h->n || v->nvec != t1->nvec || v->precision != GQT_FP64)
      return gqt::fail(GQT_ERR_ARG,
                       "%s: vectors must be FP64, of the Hamiltonian's %d sites and of one "
                       "vector count",
                       w, h->n);
  }
  const int nvec = t1->nvec;
  if (nvec != 1 && nvec != 4 && nvec != 16)
    return gqt::fail(GQT_ERR_ARG, "%s: %d vectors per call is not an FP64 form", w, nvec);
  if (out->data == t1->data)
    return gqt::fail(GQT_ERR_ARG, "%s: out must not alias t1", w);
  // The pipelined step loads the next element's left value before this element's out
  // is stored; with left == out the moment would depend on the loop shape.
  if (out->data == left->data)
    return gqt::fail(GQT_ERR_ARG, "%s: out must not alias left", w);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return gqt::cuda_fail(e, "cudaGetDevice", __FILE__, __LINE__);
  if (dev < 0 || dev >= kMaxDevices)
    return gqt::fail(GQT_ERR_ARG, "%s: device %d beyond the %d the tables hold", w, dev,
                     kMaxDevices);
  int bps = 0;
  const bool coded = h->use_codes && h->code;
  GQT_TRY(setup(dev, nvec, h->z, mode, coded, &bps));

  // Grid: as many blocks as are resident at once and as the elements need, capped so
  // that the block partials fit the static array.
  const size_t total = (size_t)h->n * nvec;
  const size_t per_block = (size_t)nvec * 4 * sizeof(double);
  size_t grid = (total + kBlock - 1) / kBlock;
  const size_t resident = (size_t)g_sms[dev] * bps;
  if (grid > resident)
    grid = resident;
  if (grid > kPartialBytes / per_block)
    grid = kPartialBytes / per_block;
  if (grid < 1)
    grid = 1;
  if (grid * per_block > kPartialBytes)
    return gqt::fail(GQT_ERR_ARG,
                     "%s: the reduction needs %zu bytes of scratch, more than the %zu bytes "
                     "of the static array",
                     w, grid * per_block, kPartialBytes);

  unsigned char* base = (unsigned char*)g_scratch_addr[dev];
  Dot d{(double*)base, (unsigned*)(base + kPartialBytes), (double2*)mu_dev};
  cudaStream_t s = gqt::stream();
  // The counter must start at zero; a previous call leaves it at zero, but clear it
  // in case that call was interrupted. The partials need no clearing: every block
  // writes its own slot before the last block reads them.
  e = cudaMemsetAsync(d.counter, 0, sizeof(unsigned), s);
  if (e != cudaSuccess)
    return gqt::cuda_fail(e, "cudaMemsetAsync(counter)", __FILE__, __LINE__);

  Op op{};  // the operator in the Hamiltonian's format (coded table or ELL arrays)
  if (coded) {
    op.code = h->code;
    op.code_delta = h->code_delta;
    op.code_hop = h->code_hop;
    op.code_xx = h->code_xx;
    op.n_codes = h->n_codes;
  }
  op.n = h->n;
  op.z = h->z;
  op.uniform = h->uniform;
  op.nn = h->nn;
  op.nl = h->nl;
  op.hop = h->hop;
  op.pot = h->pot;
  op.xx = h->xx;
  op.emax = h->energy_max;
  op.inv_emax = 1.0 / h->energy_max;
  op.lib_div = !(h->energy_max >= 0x1p-100 && h->energy_max <= 0x1p100);
  const double2* a0 = mode == 1 ? (const double2*)t0->data : nullptr;
  const double2* a1 = (const double2*)t1->data;
  double2* o = (double2*)out->data;
  const double2* l = (const double2*)left->data;
  const int g = (int)grid;
  switch (v_index(nvec)) {
    case 0:
      mode == 0 ? launch<1, kApply>(g, s, op, a0, a1, o, l, d)
                : launch<1, kCheb>(g, s, op, a0, a1, o, l, d);
      break;
    case 1:
      mode == 0 ? launch<4, kApply>(g, s, op, a0, a1, o, l, d)
                : launch<4, kCheb>(g, s, op, a0, a1, o, l, d);
      break;
    default:
      mode == 0 ? launch<16, kApply>(g, s, op, a0, a1, o, l, d)
                : launch<16, kCheb>(g, s, op, a0, a1, o, l, d);
      break;
  }
  gqt::count_launches(1);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return gqt::cuda_fail(e, "launch", __FILE__, __LINE__);
  return GQT_OK;
}
