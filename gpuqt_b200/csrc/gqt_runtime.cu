// Runtime part of the C ABI: errors, streams, device properties, vector and
// Hamiltonian handles. See include/gpuqt.h for the contract of each entry point.
#include <cstdarg>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gqt_algo.h"
#include "gqt_forms.h"
#include "gqt_internal.h"

namespace gqt {

// f(lo, hi, chunk) over [0, n) split into contiguous chunks on host threads (one
// chunk below 65,536 rows); returns the number of chunks. Chunk c covers rows
// [c * per, min(n, (c + 1) * per)).
template <class F>
int parallel_rows(long long n, F&& f)
{
  const unsigned hw = std::thread::hardware_concurrency();
  const int threads = n < (1 << 16) ? 1 : (int)std::min<unsigned>(16u, hw ? hw : 1u);
  if (threads <= 1) {
    f(0LL, n, 0);
    return 1;
  }
  const long long per = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (int c = 0; c < threads; ++c) {
    const long long lo = c * per, hi = std::min(n, lo + per);
    if (lo < hi)
      pool.emplace_back([&f, lo, hi, c] { f(lo, hi, c); });
  }
  for (auto& t : pool)
    t.join();
  return threads;
}


namespace {
thread_local std::string t_error;
thread_local cudaStream_t t_stream = nullptr;
thread_local uint64_t t_launches = 0;
}  // namespace

gqt_status fail(gqt_status code, const char* fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  t_error = buf;
  return code;
}

gqt_status cuda_fail(cudaError_t e, const char* what, const char* file, int line)
{
  return fail(e == cudaErrorMemoryAllocation ? GQT_ERR_ALLOC : GQT_ERR_CUDA,
              "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file,
              line);
}

cudaStream_t stream() { return t_stream; }

void count_launches(uint64_t k) { t_launches += k; }

const DeviceInfo& device_info()
{
  static std::mutex mu;
  static std::unordered_map<int, DeviceInfo> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it == cache.end()) {
    DeviceInfo info;
    cudaDeviceGetAttribute(&info.sms, cudaDevAttrMultiProcessorCount, dev);
    if (info.sms <= 0)
      info.sms = 1;
    it = cache.emplace(dev, info).first;
  }
  return it->second;
}

int max_grid() { return device_info().sms * (2048 / kBlock); }

int grid_for(const void* kernel, size_t total)
{
  static std::mutex mu;
  static std::unordered_map<const void*, int> per_sm;
  int bps;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = per_sm.find(kernel);
    if (it == per_sm.end()) {
      int b = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, kBlock, 0) != cudaSuccess ||
          b <= 0)
        b = 1;
      it = per_sm.emplace(kernel, b).first;
    }
    bps = it->second;
  }
  const size_t need = (total + kBlock - 1) / kBlock;
  const size_t cap = (size_t)device_info().sms * bps;
  size_t g = need < cap ? need : cap;
  if (g < 1)
    g = 1;
  const int mg = max_grid();
  return (int)(g < (size_t)mg ? g : (size_t)mg);
}

}  // namespace gqt

using namespace gqt;

namespace gqt_host {
void set_error(const std::string& message) { gqt::fail(GQT_ERR_INPUT, "%s", message.c_str()); }
}  // namespace gqt_host

// ------------------------------------------------------------------ runtime
extern "C" const char* gqt_last_error(void) { return t_error.c_str(); }

extern "C" gqt_status gqt_version(int* major, int* minor)
{
  if (major)
    *major = 1;
  if (minor)
    *minor = 0;
  return GQT_OK;
}

extern "C" gqt_status gqt_set_stream(void* s)
{
  t_stream = (cudaStream_t)s;
  return GQT_OK;
}

extern "C" void* gqt_get_stream(void) { return (void*)t_stream; }

extern "C" gqt_status gqt_sync(void)
{
  GQT_CUDA(cudaStreamSynchronize(t_stream));
  GQT_CUDA(cudaGetLastError());
  return GQT_OK;
}

extern "C" uint64_t gqt_launch_count(void) { return t_launches; }
extern "C" void gqt_reset_launch_count(void) { t_launches = 0; }

// ------------------------------------------------------------------ vectors
namespace {
gqt_status check_vec(const gqt_vec* v, const char* what)
{
  if (!v || !v->data)
    return fail(GQT_ERR_ARG, "%s: null vector", what);
  return GQT_OK;
}

gqt_status same_shape(const gqt_vec* a, const gqt_vec* b, const char* what)
{
  GQT_TRY(check_vec(a, what));
  GQT_TRY(check_vec(b, what));
  if (a->n != b->n || a->nvec != b->nvec || a->precision != b->precision)
    return fail(GQT_ERR_ARG, "%s: vectors differ in size, count or precision", what);
  return GQT_OK;
}

const FormOps* ops_of(const gqt_vec* v, const char* what)
{
  const FormOps* f = form_ops(v->precision, v->nvec);
  if (!f)
    fail(GQT_ERR_ARG, "%s: unsupported vector form (precision %d, %d vectors)", what,
         v->precision, v->nvec);
  return f;
}
}  // namespace

extern "C" gqt_status gqt_vec_create(int n, int nvec, int precision, gqt_vec** out)
{
  if (!out)
    return fail(GQT_ERR_ARG, "gqt_vec_create: null output");
  *out = nullptr;
  if (n <= 0)
    return fail(GQT_ERR_ARG, "gqt_vec_create: number of sites must be > 0 (got %d)", n);
  if (precision == GQT_FP32X || precision == GQT_FP32R || !form_ops(precision, nvec))
    return fail(GQT_ERR_ARG, "gqt_vec_create: unsupported form (precision %d, %d vectors)",
                precision, nvec);
  const size_t elem = precision == GQT_FP64 ? sizeof(double2) : sizeof(float2);
  const size_t bytes = (size_t)n * (size_t)nvec * elem;
  auto v = new (std::nothrow) gqt_vec;
  if (!v)
    return fail(GQT_ERR_ALLOC, "gqt_vec_create: host allocation failed");
  v->n = n;
  v->nvec = nvec;
  v->precision = precision;
  v->bytes = bytes;
  cudaGetDevice(&v->device);
  cudaError_t e = cudaMalloc(&v->data, bytes);
  if (e != cudaSuccess) {
    delete v;
    return cuda_fail(e, "cudaMalloc(vector)", __FILE__, __LINE__);
  }
  e = cudaMemsetAsync(v->data, 0, bytes, t_stream);
  if (e != cudaSuccess) {
    cudaFree(v->data);
    delete v;
    return cuda_fail(e, "cudaMemsetAsync(vector)", __FILE__, __LINE__);
  }
  *out = v;
  return GQT_OK;
}

extern "C" gqt_status gqt_vec_clone(const gqt_vec* src, gqt_vec** out)
{
  GQT_TRY(check_vec(src, "gqt_vec_clone"));
  GQT_TRY(gqt_vec_create(src->n, src->nvec, src->precision, out));
  GQT_CUDA(cudaMemcpyAsync((*out)->data, src->data, src->bytes, cudaMemcpyDeviceToDevice,
                           t_stream));
  return GQT_OK;
}

extern "C" gqt_status gqt_vec_destroy(gqt_vec* v)
{
  if (!v)
    return GQT_OK;
  cudaError_t e = cudaSuccess;
  if (v->data) {
    // Pending work on the current stream may still read the buffer.
    cudaStreamSynchronize(t_stream);
    e = cudaFree(v->data);
  }
  delete v;
  if (e != cudaSuccess)
    return cuda_fail(e, "cudaFree(vector)", __FILE__, __LINE__);
  return GQT_OK;
}

extern "C" gqt_status gqt_vec_info(const gqt_vec* v, int* n, int* nvec, int* precision)
{
  GQT_TRY(check_vec(v, "gqt_vec_info"));
  if (n)
    *n = v->n;
  if (nvec)
    *nvec = v->nvec;
  if (precision)
    *precision = v->precision;
  return GQT_OK;
}

extern "C" void* gqt_vec_data(gqt_vec* v) { return v ? v->data : nullptr; }

// Upload and download staging comes from a pool of this library's own that keeps its
// memory mapped between calls (release threshold: never). The default pool returns
// freed memory to the system at every synchronisation, so a loop of uploads would map
// and unmap its staging pages each time.
static gqt_status stage_alloc(double** p, size_t bytes)
{
  static std::mutex mu;
  static std::unordered_map<int, cudaMemPool_t> pools;
  int dev = 0;
  GQT_CUDA(cudaGetDevice(&dev));
  cudaMemPool_t pool;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(dev);
    if (it == pools.end()) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      GQT_CUDA(cudaMemPoolCreate(&pool, &props));
      uint64_t keep = UINT64_MAX;
      GQT_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
      it = pools.emplace(dev, pool).first;
    }
    pool = it->second;
  }
  GQT_CUDA(cudaMallocFromPoolAsync((void**)p, bytes, pool, t_stream));
  return GQT_OK;
}

extern "C" gqt_status gqt_vec_upload(gqt_vec* v, const double* re, const double* im)
{
  GQT_TRY(check_vec(v, "gqt_vec_upload"));
  if (!re || !im)
    return fail(GQT_ERR_ARG, "gqt_vec_upload: null host array");
  const FormOps* f = ops_of(v, "gqt_vec_upload");
  if (!f)
    return GQT_ERR_ARG;
  const size_t count = (size_t)v->n * v->nvec;
  double* stage = nullptr;
  GQT_TRY(stage_alloc(&stage, 2 * count * sizeof(double)));
  gqt_status st = GQT_OK;
  cudaError_t e = cudaMemcpyAsync(stage, re, count * sizeof(double), cudaMemcpyHostToDevice,
                                  t_stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(stage + count, im, count * sizeof(double), cudaMemcpyHostToDevice,
                        t_stream);
  if (e != cudaSuccess)
    st = cuda_fail(e, "cudaMemcpyAsync(upload)", __FILE__, __LINE__);
  else
    st = f->interleave(v->n, v->nvec, stage, stage + count, v->data);
  cudaFreeAsync(stage, t_stream);
  return st;
}

extern "C" gqt_status gqt_vec_download(const gqt_vec* v, double* re, double* im)
{
  GQT_TRY(check_vec(v, "gqt_vec_download"));
  if (!re || !im)
    return fail(GQT_ERR_ARG, "gqt_vec_download: null host array");
  const FormOps* f = ops_of(v, "gqt_vec_download");
  if (!f)
    return GQT_ERR_ARG;
  const size_t count = (size_t)v->n * v->nvec;
  double* stage = nullptr;
  GQT_TRY(stage_alloc(&stage, 2 * count * sizeof(double)));
  gqt_status st = f->deinterleave(v->n, v->nvec, v->data, stage, stage + count);
  if (st == GQT_OK) {
    // Through a pinned bounce buffer per device (two halves of kHalf doubles), chunk by
    // chunk: a plain DMA and a host copy, not the driver's staging path for pageable
    // memory, with the pinned memory bounded whatever the vector size. Chunk k + 1's
    // DMA into one half runs while the host copies chunk k out of the other.
    constexpr size_t kHalf = (size_t)1 << 19;  // 4 MiB
    struct Bounce {
      double* buf = nullptr;  // 2 * kHalf doubles
      cudaEvent_t done[2] = {nullptr, nullptr};
    };
    static std::mutex mu;
    static std::unordered_map<int, Bounce> bounce;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    Bounce& b = bounce[dev];
    cudaError_t e = cudaSuccess;
    if (!b.buf) {
      e = cudaMallocHost((void**)&b.buf, 2 * kHalf * sizeof(double));
      if (e != cudaSuccess)
        b.buf = nullptr;
    }
    for (int h = 0; h < 2 && e == cudaSuccess; ++h) {
      if (!b.done[h]) {
        e = cudaEventCreateWithFlags(&b.done[h], cudaEventDisableTiming);
        if (e != cudaSuccess)
          b.done[h] = nullptr;
      }
    }
    struct Chunk {
      const double* src;
      double* dst;
      size_t len;
    };
    std::vector<Chunk> chunks;
    for (int part = 0; part < 2; ++part)
      for (size_t off = 0; off < count; off += kHalf)
        chunks.push_back({stage + part * count + off, (part ? im : re) + off,
                          count - off < kHalf ? count - off : kHalf});
    auto issue = [&](size_t k) {
      const int h = (int)(k % 2);
      cudaError_t r = cudaMemcpyAsync(b.buf + h * kHalf, chunks[k].src,
                                      chunks[k].len * sizeof(double), cudaMemcpyDeviceToHost,
                                      t_stream);
      return r == cudaSuccess ? cudaEventRecord(b.done[h], t_stream) : r;
    };
    if (e == cudaSuccess && !chunks.empty())
      e = issue(0);
    for (size_t k = 0; k < chunks.size() && e == cudaSuccess; ++k) {
      // The other half's host copy (chunk k - 1) finished in the previous iteration.
      if (k + 1 < chunks.size())
        e = issue(k + 1);
      if (e == cudaSuccess)
        e = cudaEventSynchronize(b.done[k % 2]);
      if (e == cudaSuccess)
        std::memcpy(chunks[k].dst, b.buf + (k % 2) * kHalf, chunks[k].len * sizeof(double));
    }
    if (e != cudaSuccess) {
      // Leave the device's buffer usable (or absent) for the next call.
      cudaStreamSynchronize(t_stream);
      st = cuda_fail(e, "download", __FILE__, __LINE__);
    }
  }
  cudaFreeAsync(stage, t_stream);
  return st;
}

extern "C" gqt_status gqt_vec_copy(gqt_vec* dst, const gqt_vec* src)
{
  GQT_TRY(same_shape(dst, src, "gqt_vec_copy"));
  if (dst->data != src->data)
    GQT_CUDA(cudaMemcpyAsync(dst->data, src->data, src->bytes, cudaMemcpyDeviceToDevice,
                             t_stream));
  return GQT_OK;
}

extern "C" gqt_status gqt_vec_add(gqt_vec* dst, const gqt_vec* src)
{
  GQT_TRY(same_shape(dst, src, "gqt_vec_add"));
  return ops_of(dst, "gqt_vec_add")->add((size_t)dst->n * dst->nvec, dst->data, src->data);
}

extern "C" gqt_status gqt_vec_apply_sz(gqt_vec* dst, const gqt_vec* src)
{
  GQT_TRY(same_shape(dst, src, "gqt_vec_apply_sz"));
  return ops_of(dst, "gqt_vec_apply_sz")
    ->apply_sz((size_t)dst->n * dst->nvec, dst->nvec, dst->data, src->data);
}

extern "C" gqt_status gqt_vec_swap(gqt_vec* a, gqt_vec* b)
{
  GQT_TRY(same_shape(a, b, "gqt_vec_swap"));
  std::swap(a->data, b->data);
  return GQT_OK;
}

extern "C" gqt_status gqt_vec_zero(gqt_vec* v)
{
  GQT_TRY(check_vec(v, "gqt_vec_zero"));
  GQT_CUDA(cudaMemsetAsync(v->data, 0, v->bytes, t_stream));
  return GQT_OK;
}

// ------------------------------------------------------------------ Hamiltonian
gqt_ham::~gqt_ham()
{
  ws.reset();
  cudaFree(nn);
  cudaFree(nl);
  cudaFree(hop);
  cudaFree(xx);
  cudaFree(pot);
  cudaFree(pot_r);
  cudaFree(tile_first_all);  // tile_first points into it
  cudaFree(code);
  cudaFree(code_delta);
  cudaFree(code_hop);
  cudaFree(code_xx);
  cudaFree(stage_err);
  cudaFree(stage_rtab);
}

namespace {

// Host checks of one model's ELL arrays, before anything reaches the device.
gqt_status validate_desc(const gqt_ell_desc* d, const char* what)
{
  if (!d)
    return fail(GQT_ERR_ARG, "%s: null descriptor", what);
  const int n = d->n, z = d->max_neighbor;
  if (n <= 0)
    return fail(GQT_ERR_ARG, "%s: number of sites must be > 0 (got %d)", what, n);
  if (z <= 0)
    return fail(GQT_ERR_ARG, "%s: max_neighbor must be > 0 (got %d)", what, z);
  if (!(d->energy_max > 0.0))
    return fail(GQT_ERR_ARG, "%s: energy_max must be > 0 (got %g)", what, d->energy_max);
  if (!d->neighbor_number || !d->neighbor_list || !d->potential || !d->hopping_real ||
      !d->hopping_imag)
    return fail(GQT_ERR_ARG, "%s: null ELL array", what);
  if ((size_t)n * z > (size_t)1 << 40)
    return fail(GQT_ERR_ARG, "%s: n * max_neighbor too large", what);
  // The first bad row over all chunks (the one a serial scan would report).
  std::vector<long long> bad(17, -1);
  parallel_rows(n, [&](long long lo, long long hi, int chunk) {
    for (long long i = lo; i < hi; ++i) {
      const int c = d->neighbor_number[i];
      bool ok = c >= 0 && c <= z;
      for (int m = 0; ok && m < c; ++m) {
        const int j = d->neighbor_list[(size_t)i * z + m];
        ok = j >= 0 && j < n;
      }
      if (!ok) {
        bad[chunk] = i;
        return;
      }
    }
  });
  for (long long i : bad) {
    if (i < 0)
      continue;
    const int c = d->neighbor_number[i];
    if (c < 0 || c > z)
      return fail(GQT_ERR_INPUT, "%s: site %d has %d neighbours (max_neighbor %d)", what, (int)i,
                  c, z);
    for (int m = 0; m < c; ++m) {
      const int j = d->neighbor_list[(size_t)i * z + m];
      if (j < 0 || j >= n)
        return fail(GQT_ERR_INPUT, "%s: site %d neighbour %d index %d out of [0, %d)", what,
                    (int)i, m, j, n);
    }
  }
  return GQT_OK;
}

// Column-major ELL arrays of the whole (possibly batched) operator on the host.
struct Packed {
  int n = 0, z = 0;
  bool uniform = true;
  std::vector<int> nn, nl;
  std::vector<double2> hop;
  std::vector<double> xx, pot;
  void init(int n_, int z_)
  {
    n = n_;
    z = z_;
    nn.assign(n, z);
    nl.assign((size_t)n * z, 0);
    hop.assign((size_t)n * z, make_double2(0.0, 0.0));
    xx.assign((size_t)n * z, 0.0);
    pot.assign(n, 0.0);
    // Rows start as padding: full length, pointing at the site itself, zero hopping.
    parallel_rows(n, [&](long long lo, long long hi, int) {
      for (int m = 0; m < z; ++m)
        for (long long i = lo; i < hi; ++i)
          nl[(size_t)m * n + i] = (int)i;
    });
  }
};

// Copies one model into sites [base, base + d->n) of P (the transpose of
// src/hamiltonian.cu:47-88). With divide = false the values are copied bit for bit;
// with divide = true the hoppings and potentials are divided by the model's E_max.
void pack_desc(const gqt_ell_desc* d, int base, bool divide, Packed& P)
{
  const int n = d->n, z = d->max_neighbor;
  const double e = d->energy_max;
  std::atomic<bool> ragged{false};
  parallel_rows(n, [&](long long lo, long long hi, int) {
  bool short_row = false;
  for (int i = (int)lo; i < (int)hi; ++i) {
    const int c = d->neighbor_number[i];
    const int row = base + i;
    P.nn[row] = c;
    if (c != P.z)
      short_row = true;
    for (int m = 0; m < c; ++m) {
      const size_t src = (size_t)i * z + m, dst = (size_t)m * P.n + row;
      P.nl[dst] = base + d->neighbor_list[src];
      P.hop[dst] = divide ? make_double2(d->hopping_real[src] / e, d->hopping_imag[src] / e)
                          : make_double2(d->hopping_real[src], d->hopping_imag[src]);
      if (d->xx)
        P.xx[dst] = d->xx[src];
    }
    // Short rows: the entries past the row length are never read (the row length
    // bounds every loop) but point at the site itself so gathers stay in bounds.
    for (int m = c; m < P.z; ++m)
      P.nl[(size_t)m * P.n + row] = row;
    P.pot[row] = divide ? d->potential[i] / e : d->potential[i];
  }
  if (short_row)
    ragged = true;
  });
  if (ragged)
    P.uniform = false;
}

// The dictionary of (j - i, hopping, xx) over every ELL entry, padding entries
// included; false when it would exceed GQT_MAX_CODES entries.
bool build_codes(const Packed& P, std::vector<uint8_t>& codes, std::vector<int>& delta,
                 std::vector<double2>& hop, std::vector<double>& xx)
{
  struct Key {
    long long d;
    uint64_t hr, hi, x;
  };
  // At most GQT_MAX_CODES keys in first-seen order, open addressing over 1024 slots.
  struct Dict {
    std::vector<int> slot = std::vector<int>(1024, -1);
    std::vector<Key> keys;
    static uint64_t hash(const Key& k)
    {
      uint64_t h = (uint64_t)k.d * 0x9e3779b97f4a7c15ull;
      h ^= k.hr + 0x7f4a7c159e3779b9ull + (h << 6) + (h >> 2);
      h ^= k.hi + 0x94d049bb133111ebull + (h << 6) + (h >> 2);
      h ^= k.x + 0xbf58476d1ce4e5b9ull + (h << 6) + (h >> 2);
      return h ^ (h >> 29);
    }
    static bool same(const Key& a, const Key& b)
    {
      return a.d == b.d && a.hr == b.hr && a.hi == b.hi && a.x == b.x;
    }
    // The key's index, added if new; -1 once more than GQT_MAX_CODES would be kept.
    int add(const Key& k)
    {
      int s = (int)(hash(k) & 1023);
      while (slot[s] >= 0 && !same(keys[slot[s]], k))
        s = (s + 1) & 1023;
      if (slot[s] < 0) {
        if ((int)keys.size() == GQT_MAX_CODES)
          return -1;
        slot[s] = (int)keys.size();
        keys.push_back(k);
      }
      return slot[s];
    }
  };
  auto key_at = [&](int m, long long i) {
    const size_t e = (size_t)m * P.n + i;
    Key k;
    k.d = (long long)P.nl[e] - i;
    std::memcpy(&k.hr, &P.hop[e].x, 8);
    std::memcpy(&k.hi, &P.hop[e].y, 8);
    std::memcpy(&k.x, &P.xx[e], 8);
    return k;
  };
  // Pass 1: per column and chunk of rows, the keys in first-seen order; merged in the
  // order of a serial scan (column by column, rows ascending), the codes number the
  // distinct entries by first appearance whatever the chunking.
  std::atomic<bool> overflow{false};
  Dict dict;
  for (int m = 0; m < P.z && !overflow; ++m) {
    std::vector<std::vector<Key>> firsts(17);
    parallel_rows(P.n, [&](long long lo, long long hi, int chunk) {
      Dict local;
      for (long long i = lo; i < hi; ++i)
        if (local.add(key_at(m, i)) < 0) {
          overflow = true;
          return;
        }
      firsts[chunk] = std::move(local.keys);
    });
    for (auto& f : firsts)
      for (const Key& k : f)
        if (!overflow && dict.add(k) < 0)
          overflow = true;
  }
  if (overflow)
    return false;
  for (const Key& k : dict.keys) {
    double2 h;
    double x;
    std::memcpy(&h.x, &k.hr, 8);
    std::memcpy(&h.y, &k.hi, 8);
    std::memcpy(&x, &k.x, 8);
    delta.push_back((int)k.d);
    hop.push_back(h);
    xx.push_back(x);
  }
  // Pass 2: every entry's code (lookups only).
  codes.assign((size_t)P.n * P.z, 0);
  parallel_rows(P.n, [&](long long lo, long long hi, int) {
    Dict& d = dict;
    for (int m = 0; m < P.z; ++m)
      for (long long i = lo; i < hi; ++i) {
        const Key k = key_at(m, i);
        int s = (int)(Dict::hash(k) & 1023);
        while (!Dict::same(d.keys[d.slot[s]], k))
          s = (s + 1) & 1023;
        codes[(size_t)m * P.n + i] = (uint8_t)d.slot[s];
      }
  });
  return true;
}

// H = H^+ for the packed operator: for every pair of sites, the hoppings of the
// entries i -> j summed equal the conjugate of those of j -> i (relative 1e-12).
// Rows are short (z entries), so this is O(n z^2).
bool is_hermitian(const Packed& P)
{
  auto row_len = [&](int i) { return P.uniform ? P.z : P.nn[i]; };
  auto entry = [&](int i, int m) { return (size_t)m * P.n + i; };
  std::atomic<bool> broken{false};
  parallel_rows(P.n, [&](long long lo, long long hi, int) {
  for (int i = (int)lo; i < (int)hi && !broken; ++i) {
    const int ci = row_len(i);
    for (int m = 0; m < ci; ++m) {
      const int j = P.nl[entry(i, m)];
      bool first = true;  // each distinct neighbour once
      for (int q = 0; q < m; ++q)
        if (P.nl[entry(i, q)] == j)
          first = false;
      if (!first)
        continue;
      double sr = 0, si = 0, tr = 0, ti = 0, mag = 0;
      for (int q = m; q < ci; ++q)
        if (P.nl[entry(i, q)] == j) {
          sr += P.hop[entry(i, q)].x;
          si += P.hop[entry(i, q)].y;
          mag += std::fabs(P.hop[entry(i, q)].x) + std::fabs(P.hop[entry(i, q)].y);
        }
      const int cj = row_len(j);
      for (int q = 0; q < cj; ++q)
        if (P.nl[entry(j, q)] == i) {
          tr += P.hop[entry(j, q)].x;
          ti += P.hop[entry(j, q)].y;
        }
      if (j == i) {  // an entry to the site itself must be real
        if (std::fabs(si) > 1e-12 * mag)
          broken = true;
        continue;
      }
      if (std::fabs(sr - tr) > 1e-12 * mag || std::fabs(si + ti) > 1e-12 * mag)
        broken = true;
    }
  }
  });
  return !broken;
}

// Windows of the staged FP32 step (gqt_stage.cu): the neighbour offsets j - i taken by
// at least rows / 64 entries, and offset 0, grouped where consecutive offsets lie at most
// 16 rows apart; the group holding 0 first, then the most used, at most 8 in all. A
// tile of the step copies each window's rows into shared memory; entries whose offset
// lies in no window (periodic wraps, taken by a few rows per lattice line) gather from
// global memory.
struct StageWin {
  int lo, hi;
  long long use;
};

std::vector<StageWin> group_windows(const std::map<int, long long>& use, long long rows)
{
  std::vector<StageWin> wins;
  for (const auto& [d, u] : use) {
    if (d != 0 && u < rows / 64)
      continue;
    if (!wins.empty() && (long long)d - wins.back().hi <= 16) {
      wins.back().hi = d;
      wins.back().use += u;
    } else {
      wins.push_back(StageWin{d, d, u});
    }
  }
  std::stable_sort(wins.begin(), wins.end(), [](const StageWin& a, const StageWin& b) {
    const bool za = a.lo <= 0 && a.hi >= 0, zb = b.lo <= 0 && b.hi >= 0;
    if (za != zb)
      return za;
    return a.use > b.use;
  });
  if (wins.size() > (size_t)kStageWin)
    wins.resize(kStageWin);
  return wins;
}

// Entries per code over the rows [lo, hi).
std::vector<long long> code_use(const Packed& P, const std::vector<uint8_t>& codes, size_t nc,
                                long long lo, long long hi)
{
  std::vector<std::vector<long long>> part(16, std::vector<long long>(nc, 0));
  parallel_rows(hi - lo, [&](long long a, long long b, int chunk) {
    auto& u = part[chunk];
    for (int m = 0; m < P.z; ++m)
      for (long long i = lo + a; i < lo + b; ++i)
        ++u[codes[(size_t)m * P.n + i]];
  });
  std::vector<long long> use(nc, 0);
  for (auto& p : part)
    for (size_t c = 0; c < nc; ++c)
      use[c] += p[c];
  return use;
}

void plan_stage_windows(const Packed& P, const std::vector<uint8_t>& codes,
                        const std::vector<int>& delta, gqt_ham* h)
{
  static_assert(sizeof(h->stage_lo) / sizeof(int) == kStageWin, "window table size");
  const std::vector<long long> per_code = code_use(P, codes, delta.size(), 0, P.n);
  std::map<int, long long> use;  // offset -> entries
  use[0] += 0;
  for (size_t c = 0; c < delta.size(); ++c)
    use[delta[c]] += per_code[c];
  const std::vector<StageWin> wins = group_windows(use, P.n);
  h->stage_nw = (int)wins.size();
  for (size_t w = 0; w < wins.size(); ++w) {
    h->stage_lo[w] = wins[w].lo;
    h->stage_hi[w] = wins[w].hi;
  }
}

// The same per model of a realisation batch (rows [offset[r], offset[r] + n[r])), in
// common slots: slot w holds model r's w-th window, as wide as the widest of them. The
// device table gives the kernel each model's window starts and, per (model, code), the
// slot whose rows hold the code's neighbours (-1 when the model's windows miss it).
gqt_status plan_stage_windows_batch(const Packed& P, const std::vector<uint8_t>& codes,
                                    const std::vector<int>& delta,
                                    const std::vector<int>& offset,
                                    const std::vector<int>& n, gqt_ham* h)
{
  const int R = (int)n.size();
  const size_t nc = delta.size();
  std::vector<int> tab((size_t)R * (kStageWin + 1 + nc), 0);
  int* lo = tab.data();
  int* nw = lo + (size_t)R * kStageWin;
  int* slot = nw + R;
  int slots = 0;
  int width[kStageWin] = {};
  for (int r = 0; r < R; ++r) {
    const std::vector<long long> per_code = code_use(P, codes, nc, offset[r], offset[r] + n[r]);
    std::map<int, long long> use;
    use[0] += 0;
    for (size_t c = 0; c < nc; ++c)
      if (per_code[c] > 0)
        use[delta[c]] += per_code[c];
    const std::vector<StageWin> wins = group_windows(use, n[r]);
    nw[r] = (int)wins.size();
    slots = nw[r] > slots ? nw[r] : slots;
    for (int w = 0; w < nw[r]; ++w) {
      lo[(size_t)r * kStageWin + w] = wins[w].lo;
      width[w] = std::max(width[w], wins[w].hi - wins[w].lo);
    }
    for (size_t c = 0; c < nc; ++c) {
      int s = -1;
      for (int w = 0; w < nw[r] && s < 0; ++w)
        if (per_code[c] > 0 && delta[c] >= wins[w].lo && delta[c] <= wins[w].hi)
          s = w;
      slot[(size_t)r * nc + c] = s;
    }
  }
  h->stage_rnw = slots;
  for (int w = 0; w < kStageWin; ++w)
    h->stage_rwidth[w] = width[w];
  GQT_CUDA(cudaMalloc(&h->stage_rtab, tab.size() * sizeof(int)));
  GQT_CUDA(cudaMemcpy(h->stage_rtab, tab.data(), tab.size() * sizeof(int),
                      cudaMemcpyHostToDevice));
  return GQT_OK;
}

// batch_offset / batch_n: the models of a realisation batch (their staging windows are
// planned per model), or null for one model.
gqt_status upload_packed(const Packed& P, double energy_max, bool has_xx, gqt_ham* h,
                         const std::vector<int>* batch_offset = nullptr,
                         const std::vector<int>* batch_n = nullptr)
{
  const size_t pairs = (size_t)P.n * P.z;
  h->n = P.n;
  h->z = P.z;
  h->energy_max = energy_max;
  h->uniform = P.uniform ? 1 : 0;
  h->has_xx = has_xx;
  cudaGetDevice(&h->device);
  GQT_CUDA(cudaMalloc(&h->nl, pairs * sizeof(int)));
  GQT_CUDA(cudaMalloc(&h->hop, pairs * sizeof(double2)));
  GQT_CUDA(cudaMalloc(&h->xx, pairs * sizeof(double)));
  GQT_CUDA(cudaMalloc(&h->pot, (size_t)P.n * sizeof(double)));
  if (!P.uniform) {
    GQT_CUDA(cudaMalloc(&h->nn, (size_t)P.n * sizeof(int)));
    GQT_CUDA(cudaMemcpy(h->nn, P.nn.data(), (size_t)P.n * sizeof(int), cudaMemcpyHostToDevice));
  }
  GQT_CUDA(cudaMemcpy(h->nl, P.nl.data(), pairs * sizeof(int), cudaMemcpyHostToDevice));
  GQT_CUDA(cudaMemcpy(h->hop, P.hop.data(), pairs * sizeof(double2), cudaMemcpyHostToDevice));
  GQT_CUDA(cudaMemcpy(h->xx, P.xx.data(), pairs * sizeof(double), cudaMemcpyHostToDevice));
  GQT_CUDA(cudaMemcpy(h->pot, P.pot.data(), (size_t)P.n * sizeof(double),
                      cudaMemcpyHostToDevice));
  std::vector<uint8_t> codes;
  std::vector<int> delta;
  std::vector<double2> chop;
  std::vector<double> cxx;
  if (build_codes(P, codes, delta, chop, cxx)) {
    const size_t nc = delta.size();
    GQT_CUDA(cudaMalloc(&h->code, pairs));
    GQT_CUDA(cudaMalloc(&h->code_delta, nc * sizeof(int)));
    GQT_CUDA(cudaMalloc(&h->code_hop, nc * sizeof(double2)));
    GQT_CUDA(cudaMalloc(&h->code_xx, nc * sizeof(double)));
    GQT_CUDA(cudaMemcpy(h->code, codes.data(), pairs, cudaMemcpyHostToDevice));
    GQT_CUDA(cudaMemcpy(h->code_delta, delta.data(), nc * sizeof(int), cudaMemcpyHostToDevice));
    GQT_CUDA(cudaMemcpy(h->code_hop, chop.data(), nc * sizeof(double2), cudaMemcpyHostToDevice));
    GQT_CUDA(cudaMemcpy(h->code_xx, cxx.data(), nc * sizeof(double), cudaMemcpyHostToDevice));
    h->n_codes = (int)nc;
    h->use_codes = 1;
    if (batch_offset)
      GQT_TRY(plan_stage_windows_batch(P, codes, delta, *batch_offset, *batch_n, h));
    else
      plan_stage_windows(P, codes, delta, h);
    GQT_CUDA(cudaMalloc(&h->stage_err, sizeof(unsigned)));
    GQT_CUDA(cudaMemset(h->stage_err, 0, sizeof(unsigned)));
  }
  h->hermitian = is_hermitian(P) ? 1 : 0;
  h->ws.reset(new_workspace());
  return GQT_OK;
}

}  // namespace

extern "C" gqt_status gqt_ham_create(const gqt_ell_desc* d, gqt_ham** out)
{
  if (!out)
    return fail(GQT_ERR_ARG, "gqt_ham_create: null argument");
  *out = nullptr;
  if (!d)
    return fail(GQT_ERR_ARG, "gqt_ham_create: null argument");
  GQT_TRY(validate_desc(d, "gqt_ham_create"));
  Packed P;
  P.init(d->n, d->max_neighbor);
  pack_desc(d, 0, false, P);
  auto h = new (std::nothrow) gqt_ham;
  if (!h)
    return fail(GQT_ERR_ALLOC, "gqt_ham_create: host allocation failed");
  std::unique_ptr<gqt_ham> guard(h);
  GQT_TRY(upload_packed(P, d->energy_max, d->xx != nullptr, h));
  h->real_offset = {0, d->n};
  h->real_n = {d->n};
  h->real_emax = {d->energy_max};
  *out = guard.release();
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_create_batch(const gqt_ell_desc* descs, int count, gqt_ham** out)
{
  const char* w = "gqt_ham_create_batch";
  if (!out || !descs)
    return fail(GQT_ERR_ARG, "%s: null argument", w);
  *out = nullptr;
  if (count < 1 || count > GQT_MAX_REALISATIONS)
    return fail(GQT_ERR_ARG, "%s: count must be 1..%d (got %d)", w, GQT_MAX_REALISATIONS,
                count);
  const int tile = GQT_BATCH_TILE_SITES;
  long long total = 0;
  int zmax = 0;
  std::vector<int> offset(count + 1, 0);
  for (int r = 0; r < count; ++r) {
    GQT_TRY(validate_desc(&descs[r], w));
    offset[r] = (int)total;
    total += ((long long)descs[r].n + tile - 1) / tile * tile;
    zmax = descs[r].max_neighbor > zmax ? descs[r].max_neighbor : zmax;
    if (total * zmax > (long long)1 << 40 || total > 2000000000LL)
      return fail(GQT_ERR_ARG, "%s: batch too large", w);
  }
  offset[count] = (int)total;
  Packed P;
  P.init((int)total, zmax);
  for (int r = 0; r < count; ++r)
    pack_desc(&descs[r], offset[r], true, P);
  auto h = new (std::nothrow) gqt_ham;
  if (!h)
    return fail(GQT_ERR_ALLOC, "%s: host allocation failed", w);
  std::unique_ptr<gqt_ham> guard(h);
  bool has_xx = true;
  for (int r = 0; r < count; ++r)
    has_xx = has_xx && descs[r].xx != nullptr;
  // Each model is pre-divided by its own E_max, so the operator is applied with 1.
  std::vector<int> real_n(count);
  for (int r = 0; r < count; ++r)
    real_n[r] = descs[r].n;
  GQT_TRY(upload_packed(P, 1.0, has_xx, h, &offset, &real_n));
  h->n_real = count;
  h->real_offset = offset;
  for (int r = 0; r < count; ++r) {
    h->real_n.push_back(descs[r].n);
    h->real_emax.push_back(descs[r].energy_max);
  }
  // The first tile of each model for every tile size the step can run with.
  std::vector<int> first((size_t)kBatchTiles * (count + 1));
  for (int k = 0; k < kBatchTiles; ++k)
    for (int r = 0; r <= count; ++r)
      first[(size_t)k * (count + 1) + r] = offset[r] / kBatchTileSizes[k];
  GQT_CUDA(cudaMalloc(&h->tile_first_all, first.size() * sizeof(int)));
  GQT_CUDA(cudaMemcpy(h->tile_first_all, first.data(), first.size() * sizeof(int),
                      cudaMemcpyHostToDevice));
  GQT_TRY(batch_set_tile(h, kBatchTileSizes[0]));
  *out = guard.release();
  return GQT_OK;
}

namespace gqt {

gqt_status batch_set_tile(gqt_ham* h, int tile)
{
  for (int k = 0; k < kBatchTiles; ++k) {
    if (kBatchTileSizes[k] != tile)
      continue;
    if (h->tile_sites != tile && h->ws) {
      // Graphs captured so far launch the other tiling.
      cudaStreamSynchronize(t_stream);
      for (auto& kv : h->ws->graphs)
        cudaGraphExecDestroy(kv.second);
      h->ws->graphs.clear();
    }
    h->tile_sites = tile;
    h->n_tiles = h->n / tile;
    h->tile_first = h->tile_first_all + (size_t)k * (h->n_real + 1);
    return GQT_OK;
  }
  return fail(GQT_ERR_ARG, "batch tile: %d sites is not one of 256, 512, 1024", tile);
}

}  // namespace gqt

extern "C" gqt_status gqt_ham_set_batch_tile(gqt_ham* h, int tile_sites)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_set_batch_tile: null handle");
  if (h->n_real < 2 || !h->tile_first_all)
    return fail(GQT_ERR_STATE, "gqt_ham_set_batch_tile: not a realisation batch");
  return batch_set_tile(h, tile_sites);
}

extern "C" gqt_status gqt_ham_batch_tile(const gqt_ham* h, int* tile_sites)
{
  if (!h || !tile_sites)
    return fail(GQT_ERR_ARG, "gqt_ham_batch_tile: null argument");
  *tile_sites = h->n_real > 1 ? h->tile_sites : 0;
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_set_format(gqt_ham* h, int format)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_set_format: null handle");
  if (format != GQT_FORMAT_ELL && format != GQT_FORMAT_CODED)
    return fail(GQT_ERR_ARG, "gqt_ham_set_format: unknown format %d", format);
  if (format == GQT_FORMAT_CODED && !h->code)
    return fail(GQT_ERR_STATE,
                "gqt_ham_set_format: the operator has more than %d distinct entries",
                GQT_MAX_CODES);
  const int want = format == GQT_FORMAT_CODED ? 1 : 0;
  if (want != h->use_codes && h->ws) {
    // Graphs captured so far launch the other format's reads.
    cudaStreamSynchronize(t_stream);
    for (auto& kv : h->ws->graphs)
      cudaGraphExecDestroy(kv.second);
    h->ws->graphs.clear();
  }
  h->use_codes = want;
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_format(const gqt_ham* h, int* format, int* n_codes)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_format: null handle");
  if (format)
    *format = h->use_codes ? GQT_FORMAT_CODED : GQT_FORMAT_ELL;
  if (n_codes)
    *n_codes = h->n_codes;
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_realisations(const gqt_ham* h, int* count)
{
  if (!h || !count)
    return fail(GQT_ERR_ARG, "gqt_ham_realisations: null argument");
  *count = h->n_real;
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_realisation(const gqt_ham* h, int r, int* offset, int* n,
                                          double* energy_max)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_realisation: null handle");
  if (r < 0 || r >= h->n_real)
    return fail(GQT_ERR_ARG, "gqt_ham_realisation: index %d outside 0..%d", r, h->n_real - 1);
  if (offset)
    *offset = h->real_offset[r];
  if (n)
    *n = h->real_n[r];
  if (energy_max)
    *energy_max = h->real_emax[r];
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_destroy(gqt_ham* h)
{
  if (h) {
    cudaStreamSynchronize(t_stream);
    delete h;
  }
  return GQT_OK;
}

extern "C" gqt_status gqt_ham_info(const gqt_ham* h, int* n, int* z, int* uniform, double* emax)
{
  if (!h)
    return fail(GQT_ERR_ARG, "gqt_ham_info: null handle");
  if (n)
    *n = h->n;
  if (z)
    *z = h->z;
  if (uniform)
    *uniform = h->uniform;
  if (emax)
    *emax = h->energy_max;
  return GQT_OK;
}
