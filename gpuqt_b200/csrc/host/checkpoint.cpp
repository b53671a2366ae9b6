// Checkpoint file and raw moment output (see checkpoint.h).
//
// Checkpoint layout (little-endian, the host's byte order):
//   char[8]  "GQTCKPv1"
//   u64      fingerprint
//   i32 x 3  vector, stage, step
//   u64 + bytes  generator state (text)
//   u32      number of output files; per file: u64 name length, name, u64 size
//   u32      number of states; per state: u64 number of doubles, the doubles
//   u64      FNV-1a hash of everything above
#include "checkpoint.h"

#include <cstdio>
#include <cstring>
#include <fstream>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include "gpuqt.h"
#include "lsqt/model.h"

namespace gqt_host {

namespace {

const char kMagic[8] = {'G', 'Q', 'T', 'C', 'K', 'P', 'v', '1'};
const char kMomentsMagic[8] = {'G', 'Q', 'T', 'M', 'O', 'M', 'v', '1'};

uint64_t fnv1a(const void* data, size_t n, uint64_t h = 1469598103934665603ull)
{
  const unsigned char* p = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

// Flush a file, or a directory's entries (dir = true), to disk; nothing if it does not
// exist yet (an output file the run has not reached).
void sync_path(const std::string& p, bool dir)
{
  const int fd = ::open(p.c_str(), dir ? (O_RDONLY | O_DIRECTORY) : O_RDONLY);
  if (fd < 0)
    return;
  ::fsync(fd);
  ::close(fd);
}

struct Writer {
  std::string buf;
  void raw(const void* p, size_t n) { buf.append(static_cast<const char*>(p), n); }
  template <class T>
  void put(T v)
  {
    raw(&v, sizeof v);
  }
  void str(const std::string& s)
  {
    put<uint64_t>(s.size());
    raw(s.data(), s.size());
  }
};

struct Reader {
  const std::string& buf;
  size_t at = 0;
  void raw(void* p, size_t n)
  {
    if (n > buf.size() - at)
      throw InputError("checkpoint file is truncated");
    std::memcpy(p, buf.data() + at, n);
    at += n;
  }
  template <class T>
  T get()
  {
    T v;
    raw(&v, sizeof v);
    return v;
  }
  std::string str()
  {
    const uint64_t n = get<uint64_t>();
    if (n > buf.size() - at)
      throw InputError("checkpoint file is truncated");
    std::string s(buf.data() + at, n);
    at += n;
    return s;
  }
};

}  // namespace

std::string checkpoint_path(const Model& model) { return model.input_dir + "/lsqt.checkpoint"; }

uint64_t run_fingerprint(const Model& model, int precision)
{
  Writer w;
  w.put<int32_t>(model.number_of_atoms);
  w.put<int32_t>(model.max_neighbor);
  w.put<int32_t>(model.number_of_moments);
  w.put<int32_t>(model.number_of_energy_points);
  w.put<int32_t>(model.number_of_steps_correlation);
  w.put<int32_t>(model.number_of_random_vectors);
  w.put<int32_t>(model.number_of_local_orbitals);
  const int flags = (model.calculate_vac0 ? 1 : 0) | (model.calculate_vac ? 2 : 0) |
                    (model.calculate_msd ? 4 : 0) | (model.calculate_spin ? 8 : 0) |
                    (model.calculate_ldos ? 16 : 0) | (model.output_moments ? 32 : 0) |
                    (model.kpm_doubling ? 64 : 0);
  w.put<int32_t>(flags);
  w.put<int32_t>(precision);
  w.put<double>(model.energy_max);
  uint64_t h = fnv1a(w.buf.data(), w.buf.size());
  const size_t N = (size_t)model.number_of_atoms, P = N * (size_t)model.max_neighbor;
  if (model.potential)
    h = fnv1a(model.potential, N * sizeof(real), h);
  if (model.neighbor_list)
    h = fnv1a(model.neighbor_list, P * sizeof(int), h);
  if (model.hopping_real)
    h = fnv1a(model.hopping_real, P * sizeof(real), h);
  if (model.hopping_imag)
    h = fnv1a(model.hopping_imag, P * sizeof(real), h);
  if (model.energy)
    h = fnv1a(model.energy, (size_t)model.number_of_energy_points * sizeof(real), h);
  if (model.time_step)
    h = fnv1a(model.time_step, (size_t)model.number_of_steps_correlation * sizeof(real), h);
  return h;
}

std::vector<std::string> output_files(const Model& model)
{
  std::vector<std::string> f;
  auto add = [&](const char* name, bool on) {
    if (!on)
      return;
    f.push_back(std::string(name) + ".out");
    if (model.output_moments)
      f.push_back(std::string(name) + "_moments.bin");
  };
  add("dos", true);
  add("vac0", model.calculate_vac0);
  add("vac", model.calculate_vac);
  add("msd", model.calculate_msd);
  add("S", model.calculate_spin);
  add("ldos", model.calculate_ldos);
  return f;
}

void save_checkpoint(const std::string& path, const Checkpoint& ck)
{
  Writer w;
  w.raw(kMagic, sizeof kMagic);
  w.put<uint64_t>(ck.fingerprint);
  w.put<int32_t>(ck.pos.vector);
  w.put<int32_t>(ck.pos.stage);
  w.put<int32_t>(ck.pos.step);
  w.str(ck.rng);
  w.put<uint32_t>((uint32_t)ck.files.size());
  for (size_t i = 0; i < ck.files.size(); ++i) {
    w.str(ck.files[i]);
    w.put<uint64_t>(ck.sizes[i]);
  }
  w.put<uint32_t>((uint32_t)ck.states.size());
  for (const auto& s : ck.states) {
    w.put<uint64_t>(s.size());
    w.raw(s.data(), s.size() * sizeof(real));
  }
  w.put<uint64_t>(fnv1a(w.buf.data(), w.buf.size()));
  // Durable order: the output rows the checkpoint counts, then the checkpoint's own
  // bytes, then its name. A crash at any point leaves either the previous checkpoint
  // or this one, each matching output files at least as long as it records.
  const size_t slash = path.find_last_of('/');
  const std::string dir = slash == std::string::npos ? "" : path.substr(0, slash + 1);
  for (const auto& f : ck.files)
    sync_path(dir + f, false);
  const std::string tmp = path + ".tmp";
  const int fd = ::open(tmp.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
  if (fd < 0)
    die("Error: cannot write " + tmp, GQT_ERR_IO);
  size_t done = 0;
  while (done < w.buf.size()) {
    const ssize_t k = ::write(fd, w.buf.data() + done, w.buf.size() - done);
    if (k <= 0) {
      ::close(fd);
      die("Error: cannot write " + tmp, GQT_ERR_IO);
    }
    done += (size_t)k;
  }
  if (::fsync(fd) != 0) {
    ::close(fd);
    die("Error: cannot flush " + tmp + " to disk", GQT_ERR_IO);
  }
  ::close(fd);
  if (std::rename(tmp.c_str(), path.c_str()) != 0)
    die("Error: cannot rename " + tmp + " to " + path, GQT_ERR_IO);
  sync_path(dir.empty() ? "." : dir, true);
}

bool load_checkpoint(const std::string& path, Checkpoint& ck)
{
  std::ifstream in(path, std::ios::binary);
  if (!in.is_open())
    return false;
  const std::string buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  if (buf.size() < sizeof kMagic + 8 || std::memcmp(buf.data(), kMagic, sizeof kMagic) != 0)
    throw InputError(path + " is not a checkpoint of this library");
  uint64_t stored;
  std::memcpy(&stored, buf.data() + buf.size() - 8, 8);
  if (fnv1a(buf.data(), buf.size() - 8) != stored)
    throw InputError(path + " is damaged (checksum mismatch)");
  Reader r{buf};
  r.at = sizeof kMagic;
  ck.fingerprint = r.get<uint64_t>();
  ck.pos.vector = r.get<int32_t>();
  ck.pos.stage = r.get<int32_t>();
  ck.pos.step = r.get<int32_t>();
  ck.rng = r.str();
  const uint32_t nf = r.get<uint32_t>();
  ck.files.clear();
  ck.sizes.clear();
  for (uint32_t i = 0; i < nf; ++i) {
    ck.files.push_back(r.str());
    ck.sizes.push_back(r.get<uint64_t>());
  }
  const uint32_t ns = r.get<uint32_t>();
  ck.states.assign(ns, {});
  for (uint32_t i = 0; i < ns; ++i) {
    const uint64_t n = r.get<uint64_t>();
    if (n > (buf.size() - r.at) / sizeof(real))
      throw InputError(path + " is truncated");
    ck.states[i].resize(n);
    r.raw(ck.states[i].data(), n * sizeof(real));
  }
  if (r.at != buf.size() - 8)
    throw InputError(path + " has trailing data");
  return true;
}

void append_moments(const std::string& file, int n_moments, const real* re, const real* im)
{
  struct stat st;
  const bool fresh = stat(file.c_str(), &st) != 0 || st.st_size == 0;
  std::ofstream out(file, std::ios::binary | std::ios::app);
  if (!out.is_open())
    die("Error: cannot open " + file, GQT_ERR_IO);
  if (fresh) {
    const int32_t head[2] = {n_moments, 0};
    out.write(kMomentsMagic, sizeof kMomentsMagic);
    out.write(reinterpret_cast<const char*>(head), sizeof head);
  }
  std::vector<real> row(2 * (size_t)n_moments);
  for (int k = 0; k < n_moments; ++k) {
    row[2 * k] = re[k];
    row[2 * k + 1] = im[k];
  }
  out.write(reinterpret_cast<const char*>(row.data()), (std::streamsize)(row.size() * sizeof(real)));
  out.flush();
  if (!out)
    die("Error: cannot write " + file, GQT_ERR_IO);
}

}  // namespace gqt_host
