// Snapshot and checkpoint files of gadget-ng, written from the device-resident
// state or from host arrays, and read back.
//
//  * JSONL (crates/gadget-ng-io/src/snapshot.rs:124-146): meta.json,
//    provenance.json and particles.jsonl, one serde_json object per particle
//    (ParticleRecord, :17-54).  Numbers follow serde_json 1.0.149, whose f64
//    text is ryu's `format_finite`: the shortest round-trip digits (here from
//    std::to_chars) laid out in decimal while the point falls within 17 digits
//    of the first digit or at most 5 places before it, else `d.ddde-7`.
//  * bincode (crates/gadget-ng-io/src/bincode_writer.rs:16-31): the same
//    records through bincode 2.0.1's standard configuration — varint
//    integers, raw little-endian f64, the sequence length first.  A record's
//    size depends only on its global id, so every record's offset is known in
//    closed form and the device writes the whole image in parallel.
//  * checkpoint (crates/gadget-ng-cli/src/engine/checkpoint.rs:15-110):
//    checkpoint/ with the JSONL snapshot of the state and checkpoint.json.
//
// Records are written in global-id order (the order of a serial run's
// particle vector).  Velocities are the state's float32 values widened to
// f64; positions are the fixed-point positions decoded to f64.
#include <sys/stat.h>
#include <sys/types.h>

#include <algorithm>
#include <cerrno>
#include <charconv>
#include <cmath>
#include <cstring>
#include <future>
#include <string>
#include <thread>
#include <vector>

#include "../../include/treepm_b200.h"
#include "common.cuh"
#include "snapshot.cuh"
#include "tree.cuh"

namespace tpm {
namespace {

// ---- text --------------------------------------------------------------------------
// ryu's format_finite layout of the shortest round-trip digits of v.
int fmt_f64(char* out, double v) {
  if (!std::isfinite(v)) {
    std::memcpy(out, "null", 4);
    return 4;
  }
  char* o = out;
  if (std::signbit(v)) {
    *o++ = '-';
    v = -v;
  }
  if (v == 0.0) {
    std::memcpy(o, "0.0", 3);
    return (int)(o - out) + 3;
  }
  char buf[48];
  const auto r = std::to_chars(buf, buf + sizeof(buf), v, std::chars_format::scientific);
  char digits[24];
  int len = 0;
  const char* p = buf;
  while (p < r.ptr && *p != 'e') {
    if (*p != '.') digits[len++] = *p;
    ++p;
  }
  int e = 0, sgn = 1;
  if (p < r.ptr) ++p;
  if (p < r.ptr && (*p == '-' || *p == '+')) sgn = *p++ == '-' ? -1 : 1;
  while (p < r.ptr) e = e * 10 + (*p++ - '0');
  e *= sgn;
  const int kk = e + 1, k = kk - len;  // value = 0.d1..d_len x 10^kk
  if (0 <= k && kk <= 16) {
    std::memcpy(o, digits, len);
    o += len;
    std::memset(o, '0', k);
    o += k;
    *o++ = '.';
    *o++ = '0';
  } else if (0 < kk && kk <= 16) {
    std::memcpy(o, digits, kk);
    o += kk;
    *o++ = '.';
    std::memcpy(o, digits + kk, len - kk);
    o += len - kk;
  } else if (-5 < kk && kk <= 0) {
    *o++ = '0';
    *o++ = '.';
    std::memset(o, '0', -kk);
    o += -kk;
    std::memcpy(o, digits, len);
    o += len;
  } else {
    *o++ = digits[0];
    if (len > 1) {
      *o++ = '.';
      std::memcpy(o, digits + 1, len - 1);
      o += len - 1;
    }
    *o++ = 'e';
    o = std::to_chars(o, o + 8, kk - 1).ptr;
  }
  return (int)(o - out);
}

void put_f64(std::string& s, double v) {
  char b[40];
  s.append(b, fmt_f64(b, v));
}

void put_u64(std::string& s, uint64_t v) {
  char b[24];
  s.append(b, std::to_chars(b, b + sizeof(b), v).ptr - b);
}

// serde_json string escapes
void put_str(std::string& s, const char* t) {
  static const char hex[] = "0123456789abcdef";
  s.push_back('"');
  for (const unsigned char* c = (const unsigned char*)(t ? t : ""); *c; ++c) {
    switch (*c) {
      case '"': s += "\\\""; break;
      case '\\': s += "\\\\"; break;
      case '\n': s += "\\n"; break;
      case '\r': s += "\\r"; break;
      case '\t': s += "\\t"; break;
      case '\b': s += "\\b"; break;
      case '\f': s += "\\f"; break;
      default:
        if (*c < 0x20) {
          s += "\\u00";
          s.push_back(hex[*c >> 4]);
          s.push_back(hex[*c & 15]);
        } else {
          s.push_back((char)*c);
        }
    }
  }
  s.push_back('"');
}

// serde_json's pretty formatter: two spaces per level, `"key": value`.
struct Pretty {
  std::string s;
  std::vector<bool> first;
  void indent() { s.append(2 * first.size(), ' '); }
  void open(char c) {
    s.push_back(c);
    first.push_back(true);
  }
  void close(char c) {
    const bool empty = first.back();
    first.pop_back();
    if (!empty) {
      s.push_back('\n');
      indent();
    }
    s.push_back(c);
  }
  void next() {
    if (!first.back()) s.push_back(',');
    first.back() = false;
    s.push_back('\n');
    indent();
  }
  void key(const char* k) {
    next();
    put_str(s, k);
    s += ": ";
  }
  void strings(const char* const* v, int32_t n) {
    open('[');
    for (int32_t i = 0; i < n; ++i) {
      next();
      put_str(s, v[i]);
    }
    close(']');
  }
};

void pretty_provenance(Pretty& j, const tpm_provenance* p) {
  j.open('{');
  j.key("crate_version");
  put_str(j.s, p->crate_version);
  j.key("git_commit");
  if (p->git_commit)
    put_str(j.s, p->git_commit);
  else
    j.s += "null";
  j.key("build_profile");
  put_str(j.s, p->build_profile);
  j.key("enabled_features");
  j.strings(p->enabled_features, p->n_enabled_features);
  j.key("command_line");
  j.strings(p->command_line, p->n_command_line);
  j.key("config_hash");
  put_str(j.s, p->config_hash);
  j.close('}');
}

// ---- files -------------------------------------------------------------------------
void make_dirs(const std::string& dir) {
  std::string cur;
  size_t pos = 0;
  while (pos != std::string::npos) {
    pos = dir.find('/', pos + 1);
    cur = dir.substr(0, pos);
    if (cur.empty()) continue;
    if (mkdir(cur.c_str(), 0777) != 0 && errno != EEXIST)
      throw Error(TPM_ERR_IO, "cannot create " + cur + ": " + std::strerror(errno));
  }
  struct stat st;
  if (stat(dir.c_str(), &st) != 0 || !S_ISDIR(st.st_mode)) throw Error(TPM_ERR_IO, dir + " is not a directory");
}

struct File {
  FILE* f = nullptr;
  std::string path;
  File(const std::string& p, const char* mode) : path(p) {
    f = std::fopen(p.c_str(), mode);
    if (!f) throw Error(TPM_ERR_IO, "cannot open " + p + ": " + std::strerror(errno));
  }
  ~File() {
    if (f) std::fclose(f);
  }
  void write(const void* d, size_t n) {
    if (n && std::fwrite(d, 1, n, f) != n) throw Error(TPM_ERR_IO, "write to " + path + " failed");
  }
  void close() {
    FILE* g = f;
    f = nullptr;
    if (std::fclose(g) != 0) throw Error(TPM_ERR_IO, "closing " + path + " failed");
  }
};

void write_text(const std::string& path, const std::string& text) {
  File f(path, "wb");
  f.write(text.data(), text.size());
  f.close();
}

std::string read_file(const std::string& path) {
  File f(path, "rb");
  std::string s;
  char buf[1 << 16];
  size_t k;
  while ((k = std::fread(buf, 1, sizeof(buf), f.f)) > 0) s.append(buf, k);
  if (std::ferror(f.f)) throw Error(TPM_ERR_IO, "read of " + path + " failed");
  return s;
}

void write_sidecars(const std::string& dir, int64_t count, const tpm_snapshot_env* env, const tpm_provenance* prov) {
  Pretty m;
  m.open('{');
  m.key("schema_version");
  m.s += "1";
  m.key("provenance");
  pretty_provenance(m, prov);
  m.key("particle_count");
  put_u64(m.s, (uint64_t)count);
  m.key("time");
  put_f64(m.s, env->time);
  m.key("redshift");
  put_f64(m.s, env->redshift);
  m.key("box_size");
  put_f64(m.s, env->box_size);
  if (env->has_units) {
    m.key("units");
    m.open('{');
    const char* names[5] = {"length_in_kpc", "mass_in_msun", "velocity_in_km_s", "time_in_gyr", "g_internal"};
    const double vals[5] = {env->length_in_kpc, env->mass_in_msun, env->velocity_in_km_s, env->time_in_gyr,
                            env->g_internal};
    for (int i = 0; i < 5; ++i) {
      m.key(names[i]);
      put_f64(m.s, vals[i]);
    }
    m.close('}');
  }
  m.close('}');
  write_text(dir + "/meta.json", m.s);
  Pretty p;
  pretty_provenance(p, prov);
  write_text(dir + "/provenance.json", p.s);
}

unsigned host_threads() {
  const unsigned t = std::thread::hardware_concurrency();
  return std::max(1u, std::min(t ? t : 1u, 32u));
}

// Host view of a block of records: positions, velocities (n x 3), masses, ids
// (null: first_id + i).
struct HostRecords {
  const double* pos;
  const double* vel;
  const double* mass;
  const uint64_t* ids;
  uint64_t first_id;
};

void format_jsonl(const HostRecords& r, int64_t lo, int64_t hi, std::string& out) {
  out.clear();
  out.reserve((size_t)(hi - lo) * 300);
  for (int64_t i = lo; i < hi; ++i) {
    out += "{\"global_id\":";
    put_u64(out, r.ids ? r.ids[i] : r.first_id + (uint64_t)i);
    out += ",\"mass\":";
    put_f64(out, r.mass[i]);
    static const char* keys[6] = {",\"px\":", ",\"py\":", ",\"pz\":", ",\"vx\":", ",\"vy\":", ",\"vz\":"};
    for (int c = 0; c < 3; ++c) {
      out += keys[c];
      put_f64(out, r.pos[3 * i + c]);
    }
    for (int c = 0; c < 3; ++c) {
      out += keys[3 + c];
      put_f64(out, r.vel[3 * i + c]);
    }
    out += ",\"internal_energy\":0.0,\"smoothing_length\":0.0,\"ptype\":\"DarkMatter\"}\n";
  }
}

// JSONL blocks appended in order: each block is formatted by every host
// thread, then written by a background task while the next block is
// formatted (two sets of buffers).
class JsonlStream {
 public:
  explicit JsonlStream(File& f) : f_(f) {}
  ~JsonlStream() {
    if (pending_.valid()) pending_.wait();
  }
  void push(const HostRecords& r, int64_t n) {
    std::vector<std::string>& bufs = bufs_[slot_];
    const unsigned t = host_threads();
    bufs.resize(t);
    std::vector<std::thread> pool;
    for (unsigned k = 0; k < t; ++k)
      pool.emplace_back([&, k] { format_jsonl(r, n * k / t, n * (k + 1) / t, bufs[k]); });
    for (auto& th : pool) th.join();
    if (pending_.valid()) pending_.get();  // the previous block is on disk; rethrows its error
    pending_ = std::async(std::launch::async, [this, &bufs] {
      for (const std::string& b : bufs) f_.write(b.data(), b.size());
    });
    slot_ ^= 1;
  }
  void finish() {
    if (pending_.valid()) pending_.get();
  }

 private:
  File& f_;
  std::vector<std::string> bufs_[2];
  int slot_ = 0;
  std::future<void> pending_;
};

// ---- bincode ----------------------------------------------------------------------
__host__ __device__ inline int varint_size(uint64_t u) {
  return u < 251 ? 1 : u < (1ull << 16) ? 3 : u < (1ull << 32) ? 5 : 9;
}

__host__ __device__ inline int put_varint(uint8_t* o, uint64_t u) {
  const int k = varint_size(u);
  if (k == 1) {
    o[0] = (uint8_t)u;
    return 1;
  }
  o[0] = k == 3 ? 251 : k == 5 ? 252 : 253;
  for (int b = 0; b < k - 1; ++b) o[1 + b] = (uint8_t)(u >> (8 * b));
  return k;
}

// mass, px, py, pz, vx, vy, vz, internal_energy, smoothing_length, then the
// ptype variant index (one varint byte)
constexpr int REC_F64 = 9;
constexpr int REC_FIXED = REC_F64 * 8 + 1;

// Offset of the record of global id g from the first record, when the ids are
// 0..n-1 in order: the id's varint takes 1 byte below 251, 3 below 2^16, 5
// below 2^32, else 9.
__host__ __device__ inline int64_t record_offset(uint64_t g) {
  const uint64_t a = g < 251 ? g : 251, b = g < 65536 ? g : 65536, c = g < (1ull << 32) ? g : (1ull << 32);
  return (int64_t)(a * (REC_FIXED + 1) + (b > 251 ? (b - 251) * (REC_FIXED + 3) : 0) +
                   (c > 65536 ? (c - 65536) * (REC_FIXED + 5) : 0) + (g > c ? (g - c) * (REC_FIXED + 9) : 0));
}

__host__ __device__ inline int put_record(uint8_t* o, uint64_t g, double mass, const double* pos, const double* vel) {
  const int k = put_varint(o, g);
  const double f[REC_F64] = {mass, pos[0], pos[1], pos[2], vel[0], vel[1], vel[2], 0.0, 0.0};
  for (int i = 0; i < REC_F64; ++i) {
    uint64_t bits;
    memcpy(&bits, &f[i], 8);
    for (int b = 0; b < 8; ++b) o[k + 8 * i + b] = (uint8_t)(bits >> (8 * b));
  }
  o[k + 8 * REC_F64] = 0;  // ParticleType::DarkMatter
  return k + REC_FIXED;
}

// One record per thread for ids [g0, g0 + count) from id-ordered host-layout
// arrays on the device; out receives the records back to back.
__global__ void k_bincode_records(const double* __restrict__ pos, const double* __restrict__ vel,
                                  const double* __restrict__ mass, uint64_t g0, int64_t count, uint8_t* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint64_t g = g0 + (uint64_t)i;
  put_record(out + (record_offset(g) - record_offset(g0)), g, mass[g], pos + 3 * g, vel + 3 * g);
}

// The state decoded into id order: positions and velocities (n x 3) and masses.
__global__ void k_snapshot_state(Particles p, int64_t n, double scale, double* __restrict__ pos,
                                 double* __restrict__ vel, double* __restrict__ mass) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t g = p.id[i];
  pos[3 * g] = decode(p.qx[i], scale);
  pos[3 * g + 1] = decode(p.qy[i], scale);
  pos[3 * g + 2] = decode(p.qz[i], scale);
  vel[3 * g] = p.vx[i];
  vel[3 * g + 1] = p.vy[i];
  vel[3 * g + 2] = p.vz[i];
  mass[g] = p.mass[i];
}

void bincode_host(File& f, const HostRecords& r, int64_t n) {
  std::vector<uint8_t> buf;
  uint8_t hdr[9];
  f.write(hdr, put_varint(hdr, (uint64_t)n));
  const int64_t chunk = 1 << 16;
  for (int64_t lo = 0; lo < n; lo += chunk) {
    const int64_t hi = std::min(n, lo + chunk);
    buf.resize((size_t)(hi - lo) * (REC_FIXED + 9));
    size_t o = 0;
    for (int64_t i = lo; i < hi; ++i)
      o += put_record(buf.data() + o, r.ids ? r.ids[i] : r.first_id + (uint64_t)i, r.mass[i], r.pos + 3 * i,
                      r.vel + 3 * i);
    f.write(buf.data(), o);
  }
}

// ---- pinned double buffers ----------------------------------------------------------
struct Pinned {
  void* p = nullptr;
  explicit Pinned(size_t bytes) { TPM_CUDA(cudaMallocHost(&p, bytes)); }
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

struct DeviceBuf {
  void* p = nullptr;
  explicit DeviceBuf(size_t bytes) { TPM_CUDA(cudaMalloc(&p, bytes)); }
  ~DeviceBuf() {
    if (p) cudaFree(p);
  }
};

struct Event {
  cudaEvent_t e = nullptr;
  Event() { TPM_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)); }
  ~Event() {
    if (e) cudaEventDestroy(e);
  }
};

// ---- reading --------------------------------------------------------------------------
struct Parsed {
  std::vector<double> pos, vel, mass;
  std::vector<uint64_t> ids;
};

const char* skip_ws(const char* p, const char* e) {
  while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
  return p;
}

// One JSONL object: the fields of ParticleRecord in any order; unknown keys
// with string, number, true/false/null values are skipped.
bool parse_record(const char* p, const char* e, uint64_t* id, double f[7]) {
  static const char* names[7] = {"mass", "px", "py", "pz", "vx", "vy", "vz"};
  int seen = 0;
  p = skip_ws(p, e);
  if (p >= e || *p++ != '{') return false;
  for (;;) {
    p = skip_ws(p, e);
    if (p < e && *p == '}') break;
    if (p >= e || *p != '"') return false;
    const char* k0 = ++p;
    while (p < e && *p != '"') p += (*p == '\\') ? 2 : 1;
    if (p >= e) return false;
    const std::string key(k0, p - k0);
    p = skip_ws(p + 1, e);
    if (p >= e || *p++ != ':') return false;
    p = skip_ws(p, e);
    if (key == "global_id") {
      auto r = std::from_chars(p, e, *id);
      if (r.ec != std::errc()) return false;
      p = r.ptr;
      seen |= 1 << 7;
    } else {
      int which = -1;
      for (int i = 0; i < 7; ++i)
        if (key == names[i]) which = i;
      if (which >= 0) {
        auto r = std::from_chars(p, e, f[which]);
        if (r.ec != std::errc()) return false;
        p = r.ptr;
        seen |= 1 << which;
      } else if (p < e && *p == '"') {
        ++p;
        while (p < e && *p != '"') p += (*p == '\\') ? 2 : 1;
        ++p;
      } else {
        while (p < e && *p != ',' && *p != '}') ++p;
      }
    }
    p = skip_ws(p, e);
    if (p < e && *p == ',') {
      ++p;
      continue;
    }
    if (p < e && *p == '}') break;
    return false;
  }
  return seen == 0xFF;
}

Parsed parse_jsonl(const std::string& text) {
  std::vector<int64_t> starts;
  for (size_t i = 0; i < text.size();) {
    size_t j = text.find('\n', i);
    if (j == std::string::npos) j = text.size();
    const char* b = skip_ws(text.data() + i, text.data() + j);
    if (b < text.data() + j) starts.push_back((int64_t)i);
    i = j + 1;
  }
  const int64_t n = (int64_t)starts.size();
  Parsed out;
  out.pos.resize(3 * n);
  out.vel.resize(3 * n);
  out.mass.resize(n);
  out.ids.resize(n);
  const unsigned t = host_threads();
  std::vector<int64_t> bad(t, -1);
  std::vector<std::thread> pool;
  for (unsigned k = 0; k < t; ++k)
    pool.emplace_back([&, k] {
      for (int64_t r = n * k / t; r < n * (k + 1) / t; ++r) {
        const char* b = text.data() + starts[r];
        const char* e = (const char*)std::memchr(b, '\n', text.data() + text.size() - b);
        if (!e) e = text.data() + text.size();
        double f[7];
        uint64_t g = 0;
        if (!parse_record(b, e, &g, f)) {
          bad[k] = r;
          return;
        }
        out.ids[r] = g;
        out.mass[r] = f[0];
        for (int c = 0; c < 3; ++c) {
          out.pos[3 * r + c] = f[1 + c];
          out.vel[3 * r + c] = f[4 + c];
        }
      }
    });
  for (auto& th : pool) th.join();
  for (int64_t b : bad)
    if (b >= 0) throw Error(TPM_ERR_IO, "malformed particle record on line " + std::to_string(b + 1));
  return out;
}

Parsed parse_bincode(const std::string& d) {
  size_t o = 0;
  auto rd = [&](uint64_t* v) {
    if (o >= d.size()) return false;
    const uint8_t b = (uint8_t)d[o];
    const int k = b < 251 ? 1 : b == 251 ? 3 : b == 252 ? 5 : b == 253 ? 9 : 0;
    if (k == 0 || o + k > d.size()) return false;
    uint64_t u = 0;
    if (k == 1)
      u = b;
    else
      for (int i = 0; i < k - 1; ++i) u |= (uint64_t)(uint8_t)d[o + 1 + i] << (8 * i);
    o += k;
    *v = u;
    return true;
  };
  uint64_t n = 0;
  if (!rd(&n) || n > d.size()) throw Error(TPM_ERR_IO, "malformed particles.bin header");
  Parsed out;
  out.pos.resize(3 * n);
  out.vel.resize(3 * n);
  out.mass.resize(n);
  out.ids.resize(n);
  for (uint64_t r = 0; r < n; ++r) {
    uint64_t g, t;
    if (!rd(&g) || o + 8 * REC_F64 > d.size()) throw Error(TPM_ERR_IO, "truncated particles.bin");
    double f[REC_F64];
    std::memcpy(f, d.data() + o, 8 * REC_F64);
    o += 8 * REC_F64;
    if (!rd(&t) || t > 2) throw Error(TPM_ERR_IO, "bad particle type in particles.bin");
    out.ids[r] = g;
    out.mass[r] = f[0];
    for (int c = 0; c < 3; ++c) {
      out.pos[3 * r + c] = f[1 + c];
      out.vel[3 * r + c] = f[4 + c];
    }
  }
  if (o != d.size()) throw Error(TPM_ERR_IO, "trailing bytes in particles.bin");
  return out;
}

// Value of a top-level number (or string) key of a small JSON file.
bool json_number(const std::string& s, const char* key, double* v) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = s.find(k);
  if (p == std::string::npos) return false;
  p = s.find(':', p + k.size());
  if (p == std::string::npos) return false;
  const char* b = skip_ws(s.data() + p + 1, s.data() + s.size());
  while (b < s.data() + s.size() && *b == '\n') b = skip_ws(b + 1, s.data() + s.size());
  return std::from_chars(b, s.data() + s.size(), *v).ec == std::errc();
}

bool json_string_value(const std::string& s, const char* key, std::string* v) {
  const std::string k = std::string("\"") + key + "\"";
  size_t p = s.find(k);
  if (p == std::string::npos) return false;
  p = s.find('"', s.find(':', p + k.size()));
  if (p == std::string::npos) return false;
  const size_t q = s.find('"', p + 1);
  if (q == std::string::npos) return false;
  *v = s.substr(p + 1, q - p - 1);
  return true;
}

}  // namespace

// ---- entry points used by the handle API ------------------------------------------------
void snapshot_write(const std::string& dir, int32_t format, const tpm_snapshot_env* env, const tpm_provenance* prov,
                    const DeviceState& st) {
  if (format != TPM_SNAPSHOT_JSONL && format != TPM_SNAPSHOT_BINCODE)
    throw Error(TPM_ERR_INVALID_ARGUMENT, "unknown snapshot format");
  make_dirs(dir);
  write_sidecars(dir, st.n, env, prov);
  const int64_t n = st.n;
  cudaStream_t s = st.stream;
  double* dpos = st.staging;
  double* dvel = st.staging + 3 * n;
  double* dmass = st.staging + 6 * n;
  if (n > 0) {
    k_snapshot_state<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(st.p, n, st.box / TWO32, dpos, dvel, dmass);
    TPM_LAUNCH_CHECK();
  }
  const int64_t chunk = std::min<int64_t>(std::max<int64_t>(n, 1), 1 << 20);
  if (format == TPM_SNAPSHOT_JSONL) {
    File f(dir + "/particles.jsonl", "wb");
    // per buffer: chunk x (3 + 3 + 1) doubles; copy chunk c + 1 while chunk c is formatted
    Pinned host(2 * (size_t)chunk * 7 * sizeof(double));
    Event ev[2];
    JsonlStream js(f);
    auto issue = [&](int64_t lo, int slot) {
      const int64_t m = std::min(chunk, n - lo);
      double* h = (double*)host.p + (size_t)slot * chunk * 7;
      TPM_CUDA(cudaMemcpyAsync(h, dpos + 3 * lo, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaMemcpyAsync(h + 3 * chunk, dvel + 3 * lo, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaMemcpyAsync(h + 6 * chunk, dmass + lo, sizeof(double) * m, cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaEventRecord(ev[slot].e, s));
    };
    if (n > 0) issue(0, 0);
    for (int64_t lo = 0, c = 0; lo < n; lo += chunk, ++c) {
      const int slot = (int)(c & 1);
      TPM_CUDA(cudaEventSynchronize(ev[slot].e));
      if (lo + chunk < n) issue(lo + chunk, slot ^ 1);
      const double* h = (const double*)host.p + (size_t)slot * chunk * 7;
      const HostRecords r{h, h + 3 * chunk, h + 6 * chunk, nullptr, (uint64_t)lo};
      js.push(r, std::min(chunk, n - lo));
    }
    js.finish();
    f.close();
  } else {
    File f(dir + "/particles.bin", "wb");
    uint8_t hdr[9];
    f.write(hdr, put_varint(hdr, (uint64_t)n));
    const size_t max_bytes = (size_t)chunk * (REC_FIXED + 9);
    DeviceBuf dev(2 * max_bytes);
    Pinned host(2 * max_bytes);
    Event ev[2];
    size_t bytes[2] = {0, 0};
    auto issue = [&](int64_t lo, int slot) {
      const int64_t m = std::min(chunk, n - lo);
      uint8_t* d = (uint8_t*)dev.p + slot * max_bytes;
      k_bincode_records<<<grid_for(m, 256, 1ll << 30), 256, 0, s>>>(dpos, dvel, dmass, (uint64_t)lo, m, d);
      TPM_LAUNCH_CHECK();
      bytes[slot] = (size_t)(record_offset((uint64_t)(lo + m)) - record_offset((uint64_t)lo));
      TPM_CUDA(cudaMemcpyAsync((uint8_t*)host.p + slot * max_bytes, d, bytes[slot], cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaEventRecord(ev[slot].e, s));
    };
    if (n > 0) issue(0, 0);
    for (int64_t lo = 0, c = 0; lo < n; lo += chunk, ++c) {
      const int slot = (int)(c & 1);
      TPM_CUDA(cudaEventSynchronize(ev[slot].e));
      const size_t here = bytes[slot];
      if (lo + chunk < n) issue(lo + chunk, slot ^ 1);
      f.write((uint8_t*)host.p + slot * max_bytes, here);
    }
    f.close();
  }
  TPM_CUDA(cudaStreamSynchronize(s));
}

void snapshot_write_host(const std::string& dir, int32_t format, const double* pos, const double* vel,
                         const double* mass, const uint64_t* ids, int64_t n, const tpm_snapshot_env* env,
                         const tpm_provenance* prov) {
  if (format != TPM_SNAPSHOT_JSONL && format != TPM_SNAPSHOT_BINCODE)
    throw Error(TPM_ERR_INVALID_ARGUMENT, "unknown snapshot format");
  make_dirs(dir);
  write_sidecars(dir, n, env, prov);
  const HostRecords r{pos, vel, mass, ids, 0};
  if (format == TPM_SNAPSHOT_JSONL) {
    File f(dir + "/particles.jsonl", "wb");
    JsonlStream js(f);
    const int64_t chunk = 1 << 20;
    for (int64_t lo = 0; lo < n; lo += chunk) {
      const HostRecords c{pos + 3 * lo, vel + 3 * lo, mass + lo, ids ? ids + lo : nullptr, (uint64_t)lo};
      js.push(c, std::min(chunk, n - lo));
    }
    js.finish();
    f.close();
  } else {
    File f(dir + "/particles.bin", "wb");
    bincode_host(f, r, n);
    f.close();
  }
}

void snapshot_read(const std::string& dir, int32_t format, tpm_snapshot_env* env, std::vector<double>& pos,
                   std::vector<double>& vel, std::vector<double>& mass, std::vector<uint64_t>& ids) {
  if (format != TPM_SNAPSHOT_JSONL && format != TPM_SNAPSHOT_BINCODE)
    throw Error(TPM_ERR_INVALID_ARGUMENT, "unknown snapshot format");
  Parsed p = format == TPM_SNAPSHOT_JSONL ? parse_jsonl(read_file(dir + "/particles.jsonl"))
                                          : parse_bincode(read_file(dir + "/particles.bin"));
  if (env) {
    const std::string meta = read_file(dir + "/meta.json");
    *env = tpm_snapshot_env{};
    if (!json_number(meta, "time", &env->time) || !json_number(meta, "redshift", &env->redshift) ||
        !json_number(meta, "box_size", &env->box_size))
      throw Error(TPM_ERR_IO, "meta.json lacks time, redshift or box_size");
    if (meta.find("\"units\"") != std::string::npos) {
      env->has_units = 1;
      json_number(meta, "length_in_kpc", &env->length_in_kpc);
      json_number(meta, "mass_in_msun", &env->mass_in_msun);
      json_number(meta, "velocity_in_km_s", &env->velocity_in_km_s);
      json_number(meta, "time_in_gyr", &env->time_in_gyr);
      json_number(meta, "g_internal", &env->g_internal);
    }
  }
  pos.swap(p.pos);
  vel.swap(p.vel);
  mass.swap(p.mass);
  ids.swap(p.ids);
}

// Records in global-id order (ids must be a permutation of 0..n-1).
void order_by_id(std::vector<double>& pos, std::vector<double>& vel, std::vector<double>& mass,
                 const std::vector<uint64_t>& ids) {
  const size_t n = ids.size();
  std::vector<double> p2(3 * n), v2(3 * n), m2(n);
  std::vector<uint8_t> seen(n, 0);
  for (size_t r = 0; r < n; ++r) {
    const uint64_t g = ids[r];
    if (g >= n || seen[g]) throw Error(TPM_ERR_IO, "global ids are not a permutation of 0..n-1");
    seen[g] = 1;
    for (int c = 0; c < 3; ++c) {
      p2[3 * g + c] = pos[3 * r + c];
      v2[3 * g + c] = vel[3 * r + c];
    }
    m2[g] = mass[r];
  }
  pos.swap(p2);
  vel.swap(v2);
  mass.swap(m2);
}

void checkpoint_write_meta(const std::string& ck_dir, uint64_t completed_step, double a_current,
                           const char* config_hash, int64_t total) {
  Pretty j;
  j.open('{');
  j.key("schema_version");
  j.s += "1";
  j.key("completed_step");
  put_u64(j.s, completed_step);
  j.key("a_current");
  put_f64(j.s, a_current);
  j.key("config_hash");
  put_str(j.s, config_hash);
  j.key("total_particles");
  put_u64(j.s, (uint64_t)total);
  for (const char* k : {"has_hierarchical_state", "sfc_state_saved", "has_agn_state", "has_chem_state"}) {
    j.key(k);
    j.s += "false";
  }
  j.close('}');
  write_text(ck_dir + "/checkpoint.json", j.s);
}

void checkpoint_read_meta(const std::string& ck_dir, uint64_t* completed_step, double* a_current,
                          std::string* config_hash, int64_t* total) {
  const std::string s = read_file(ck_dir + "/checkpoint.json");
  double step = 0.0, tot = 0.0;
  if (!json_number(s, "completed_step", &step) || !json_number(s, "a_current", a_current) ||
      !json_string_value(s, "config_hash", config_hash) || !json_number(s, "total_particles", &tot))
    throw Error(TPM_ERR_IO, "checkpoint.json lacks completed_step, a_current, config_hash or total_particles");
  *completed_step = (uint64_t)step;
  *total = (int64_t)tot;
}

}  // namespace tpm

// ---- host-array C ABI (no device needed) ----------------------------------------------------
namespace {
thread_local std::string g_snapshot_error;
}

extern "C" const char* tpm_snapshot_last_error(void) { return g_snapshot_error.c_str(); }

extern "C" int tpm_write_snapshot_host(const char* out_dir, int32_t format, const double* pos, const double* vel,
                                       const double* mass, const uint64_t* global_ids, int64_t n,
                                       const tpm_snapshot_env* env, const tpm_provenance* prov) {
  if (!out_dir || !env || !prov || n < 0 || (n > 0 && (!pos || !vel || !mass))) return TPM_ERR_INVALID_ARGUMENT;
  try {
    tpm::snapshot_write_host(out_dir, format, pos, vel, mass, global_ids, n, env, prov);
  } catch (const tpm::Error& e) {
    g_snapshot_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_snapshot_error = e.what();
    return TPM_ERR_IO;
  }
  return TPM_OK;
}

extern "C" int tpm_read_snapshot_host(const char* dir, int32_t format, int64_t* n_out, double* pos, double* vel,
                                      double* mass, uint64_t* global_ids, int64_t capacity,
                                      tpm_snapshot_env* env_out) {
  if (!dir || !n_out) return TPM_ERR_INVALID_ARGUMENT;
  try {
    std::vector<double> p, v, m;
    std::vector<uint64_t> ids;
    tpm::snapshot_read(dir, format, env_out, p, v, m, ids);
    const int64_t n = (int64_t)ids.size();
    *n_out = n;
    if (pos || vel || mass || global_ids) {
      if (capacity < n) return TPM_ERR_INVALID_ARGUMENT;
      if (pos) std::memcpy(pos, p.data(), sizeof(double) * 3 * n);
      if (vel) std::memcpy(vel, v.data(), sizeof(double) * 3 * n);
      if (mass) std::memcpy(mass, m.data(), sizeof(double) * n);
      if (global_ids) std::memcpy(global_ids, ids.data(), sizeof(uint64_t) * n);
    }
  } catch (const tpm::Error& e) {
    g_snapshot_error = e.what();
    return e.code;
  } catch (const std::exception& e) {
    g_snapshot_error = e.what();
    return TPM_ERR_IO;
  }
  return TPM_OK;
}
