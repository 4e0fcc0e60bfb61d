// Manifest graph format: reader, device loader, writer.
//
// Reference: kaspan/scc/adapter/manifest.hpp:19-198 (the text manifest:
// one `key value` per line, `%` comment lines, the keys listed in
// kspn_manifest_read) and :200-245 (load_graph_from_manifest: four files of
// dense unsigned integers, graph.head.bytes / graph.csr.bytes bytes each
// (1..8), in graph.endian byte order; head n + 1 entries, csr m entries).
//
// On the device: each file is read into a pinned host chunk (two chunks,
// so reading the next chunk overlaps the copy and decode of the last),
// copied as raw bytes, and a kernel widens (or narrows) every entry to the
// library's types (u64 offsets, u32 ids), swapping byte order when asked.
// Entries that do not fit the target type are counted and reported.
#include "kspn_internal.cuh"

#include <cerrno>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

namespace kspn {

namespace {

// raw[i * w .. i * w + w) as an unsigned integer (big: most significant
// byte first) into out[i]; entries above `limit` counted in *bad
template<typename T>
__global__ void
k_decode(uint8_t const* __restrict__ raw, uint64_t count, uint32_t w, int big, uint64_t limit, T* __restrict__ out, uint32_t* bad)
{
  uint32_t nbad = 0;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
    uint8_t const* p = raw + i * w;
    uint64_t       v = 0;
    if (big)
      for (uint32_t b = 0; b < w; ++b) v = (v << 8) | p[b];
    else
      for (uint32_t b = w; b-- > 0;) v = (v << 8) | p[b];
    if (v > limit) ++nbad;
    out[i] = static_cast<T>(v);
  }
  if (nbad) atomicAdd(bad, nbad);
}

struct pinned
{
  void* p = nullptr;
  ~pinned()
  {
    if (p) cudaFreeHost(p);
  }
};

// One file of `count` entries of `w` bytes into dev[0, count).
template<typename T>
void
load_file(kspn_context* ctx, std::string const& path, uint64_t count, uint32_t w, bool big, uint64_t limit, T* dev, uint8_t* stage, void* const (&host)[2], size_t chunk_entries)
{
  std::FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: cannot open " + path + ": " + std::strerror(errno) };
  struct closer
  {
    std::FILE* f;
    ~closer() { std::fclose(f); }
  } guard_f{ f };
  cudaStream_t const s = ctx->stream;
  uint32_t* const    bad = ctx->ws.ctr + CTR_ERR;
  KSPN_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), s));
  int k = 0;
  for (uint64_t done = 0; done < count; k ^= 1) {
    uint64_t const n = count - done < chunk_entries ? count - done : chunk_entries;
    // the copy that last used this host chunk has finished
    KSPN_CUDA(cudaEventSynchronize(ctx->pe[k]));
    size_t const got = std::fread(host[k], w, n, f);
    if (got != n) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: " + path + " is shorter than its manifest says" };
    uint8_t* const st = stage + static_cast<size_t>(k) * chunk_entries * 8;
    KSPN_CUDA(cudaMemcpyAsync(st, host[k], n * w, cudaMemcpyHostToDevice, s));
    KSPN_CUDA(cudaEventRecord(ctx->pe[k], s));
    uint64_t const b = (n + 255) / 256;
    k_decode<T><<<static_cast<unsigned>(b < 148ull * 16 ? b : 148ull * 16), 256, 0, s>>>(st, n, w, big ? 1 : 0, limit, dev + done, bad);
    KSPN_CHECK_LAUNCH();
    ctx->launches += 1;
    done += n;
  }
  uint32_t h = 0;
  KSPN_CUDA(cudaMemcpyAsync(&h, bad, sizeof(h), cudaMemcpyDeviceToHost, s));
  KSPN_CUDA(cudaStreamSynchronize(s));
  if (h) throw error{ KSPN_ERR_INVALID_GRAPH, "manifest: " + std::to_string(h) + " entries of " + path + " are out of range" };
}

void
copy_str(char* dst, size_t cap, std::string const& s)
{
  if (s.size() >= cap) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: value too long: " + s };
  std::memcpy(dst, s.c_str(), s.size() + 1);
}

uint64_t
parse_u64(std::string const& key, std::string const& v)
{
  if (v.empty()) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: " + key + " is empty" };
  uint64_t x = 0;
  for (char c : v) {
    if (c < '0' || c > '9') throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: " + key + " is not an unsigned integer: " + v };
    uint64_t const y = x * 10 + static_cast<uint64_t>(c - '0');
    if (y / 10 != x) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: " + key + " overflows: " + v };
    x = y;
  }
  return x;
}

int
parse_bool(std::string const& key, std::string const& v)
{
  if (v == "true") return 1;
  if (v == "false") return 0;
  throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: " + key + " must be true or false: " + v };
}

std::string
dir_of(std::string const& path)
{
  size_t const i = path.find_last_of('/');
  return i == std::string::npos ? std::string(".") : path.substr(0, i);
}

} // namespace

void
manifest_read(char const* path, kspn_manifest* out)
{
  std::ifstream in(path);
  if (!in.is_open()) throw error{ KSPN_ERR_INVALID_ARGUMENT, std::string("manifest: cannot open ") + path };
  std::map<std::string, std::string> kv;
  std::string                        line;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty() || line[0] == '%') continue;
    size_t const key_end = line.find(' ');
    if (key_end == std::string::npos) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: line without a value: " + line };
    size_t v = key_end;
    while (v < line.size() && line[v] == ' ') ++v;
    if (!kv.emplace(line.substr(0, key_end), line.substr(v)).second) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: duplicate key " + line.substr(0, key_end) };
  }
  auto get = [&](char const* key) -> std::string const& {
    auto it = kv.find(key);
    if (it == kv.end()) throw error{ KSPN_ERR_INVALID_ARGUMENT, std::string("manifest: missing key ") + key };
    return it->second;
  };
  std::memset(out, 0, sizeof(*out));
  out->schema_version = static_cast<uint32_t>(parse_u64("schema.version", get("schema.version")));
  copy_str(out->graph_code, sizeof(out->graph_code), get("graph.code"));
  copy_str(out->graph_name, sizeof(out->graph_name), get("graph.name"));
  std::string const& e = get("graph.endian");
  if (e == "little") out->big_endian = 0;
  else if (e == "big") out->big_endian = 1;
  else throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: graph.endian must be little or big: " + e };
  out->node_count      = parse_u64("graph.node_count", get("graph.node_count"));
  out->edge_count      = parse_u64("graph.edge_count", get("graph.edge_count"));
  out->self_loops      = parse_bool("graph.contains_self_loops", get("graph.contains_self_loops"));
  out->duplicate_edges = parse_bool("graph.contains_duplicate_edges", get("graph.contains_duplicate_edges"));
  out->head_bytes      = static_cast<uint32_t>(parse_u64("graph.head.bytes", get("graph.head.bytes")));
  out->csr_bytes       = static_cast<uint32_t>(parse_u64("graph.csr.bytes", get("graph.csr.bytes")));
  if (out->head_bytes < 1 || out->head_bytes > 8 || out->csr_bytes < 1 || out->csr_bytes > 8) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: entry widths must be 1..8 bytes" };
  std::string const base = dir_of(path) + "/";
  copy_str(out->fw_head_path, sizeof(out->fw_head_path), base + get("fw.head.path"));
  copy_str(out->fw_csr_path, sizeof(out->fw_csr_path), base + get("fw.csr.path"));
  copy_str(out->bw_head_path, sizeof(out->bw_head_path), base + get("bw.head.path"));
  copy_str(out->bw_csr_path, sizeof(out->bw_csr_path), base + get("bw.csr.path"));
}

void
manifest_load(kspn_context* ctx, kspn_manifest const& mf, uint64_t* fh, uint32_t* fc, uint64_t* bh, uint32_t* bc)
{
  uint64_t const n = mf.node_count, m = mf.edge_count;
  if (n >= 0xFFFFFFFFull) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: node_count must be below 2^32 - 1" };
  ensure_workspace(ctx, 1, 0); // counters
  size_t const chunk = 32ull << 20; // entries per chunk
  size_t const maxw  = mf.head_bytes > mf.csr_bytes ? mf.head_bytes : mf.csr_bytes;
  pinned       h0, h1;
  KSPN_CUDA(cudaMallocHost(&h0.p, chunk * maxw));
  KSPN_CUDA(cudaMallocHost(&h1.p, chunk * maxw));
  void* const host[2] = { h0.p, h1.p };
  auto* const stage   = static_cast<uint8_t*>(context_buffer(ctx, BUF_BUILD, 2 * chunk * 8));
  KSPN_CUDA(cudaEventRecord(ctx->pe[0], ctx->stream));
  KSPN_CUDA(cudaEventRecord(ctx->pe[1], ctx->stream));
  bool const big = mf.big_endian != 0;
  load_file<uint64_t>(ctx, mf.fw_head_path, n + 1, mf.head_bytes, big, m, fh, stage, host, chunk);
  if (m) load_file<uint32_t>(ctx, mf.fw_csr_path, m, mf.csr_bytes, big, n ? n - 1 : 0, fc, stage, host, chunk);
  load_file<uint64_t>(ctx, mf.bw_head_path, n + 1, mf.head_bytes, big, m, bh, stage, host, chunk);
  if (m) load_file<uint32_t>(ctx, mf.bw_csr_path, m, mf.csr_bytes, big, n ? n - 1 : 0, bc, stage, host, chunk);
}

namespace {

void
write_file(std::string const& path, void const* data, uint64_t count, uint32_t src_bytes, uint32_t w, bool big)
{
  std::FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: cannot create " + path };
  std::string buf;
  buf.resize(static_cast<size_t>(1) << 20);
  size_t     pos = 0;
  bool       ok  = true;
  auto const* src = static_cast<uint8_t const*>(data);
  for (uint64_t i = 0; i < count; ++i) {
    uint64_t v = 0;
    std::memcpy(&v, src + i * src_bytes, src_bytes); // the host is little-endian
    if (w < 8 && (v >> (8 * w)) != 0) {
      std::fclose(f);
      throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: an entry does not fit " + std::to_string(w) + " bytes" };
    }
    for (uint32_t b = 0; b < w; ++b) buf[pos + b] = static_cast<char>((v >> (8 * (big ? w - 1 - b : b))) & 0xFF);
    pos += w;
    if (pos + 8 > buf.size()) {
      ok  = ok && std::fwrite(buf.data(), 1, pos, f) == pos;
      pos = 0;
    }
  }
  ok = ok && std::fwrite(buf.data(), 1, pos, f) == pos;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: cannot write " + path };
}

} // namespace

void
manifest_write(char const* dir, char const* name, uint32_t n, uint64_t m, uint64_t const* fh, uint32_t const* fc, uint64_t const* bh, uint32_t const* bc, uint32_t head_bytes, uint32_t csr_bytes,
               int big_endian, int self_loops, int duplicate_edges)
{
  if (head_bytes < 1 || head_bytes > 8 || csr_bytes < 1 || csr_bytes > 8) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: entry widths must be 1..8 bytes" };
  std::string const d = dir, nm = name;
  write_file(d + "/" + nm + ".fw.head.bin", fh, static_cast<uint64_t>(n) + 1, 8, head_bytes, big_endian != 0);
  write_file(d + "/" + nm + ".fw.csr.bin", fc, m, 4, csr_bytes, big_endian != 0);
  write_file(d + "/" + nm + ".bw.head.bin", bh, static_cast<uint64_t>(n) + 1, 8, head_bytes, big_endian != 0);
  write_file(d + "/" + nm + ".bw.csr.bin", bc, m, 4, csr_bytes, big_endian != 0);
  std::ofstream out(d + "/" + nm + ".manifest");
  out << "% written by kspn_manifest_write\n"
      << "schema.version 1\n"
      << "graph.code " << nm << "\n"
      << "graph.name " << nm << "\n"
      << "graph.endian " << (big_endian ? "big" : "little") << "\n"
      << "graph.node_count " << n << "\n"
      << "graph.edge_count " << m << "\n"
      << "graph.contains_self_loops " << (self_loops ? "true" : "false") << "\n"
      << "graph.contains_duplicate_edges " << (duplicate_edges ? "true" : "false") << "\n"
      << "graph.head.bytes " << head_bytes << "\n"
      << "graph.csr.bytes " << csr_bytes << "\n"
      << "fw.head.path " << nm << ".fw.head.bin\n"
      << "fw.csr.path " << nm << ".fw.csr.bin\n"
      << "bw.head.path " << nm << ".bw.head.bin\n"
      << "bw.csr.path " << nm << ".bw.csr.bin\n";
  if (!out.good()) throw error{ KSPN_ERR_INVALID_ARGUMENT, "manifest: cannot write " + d + "/" + nm + ".manifest" };
}

} // namespace kspn
