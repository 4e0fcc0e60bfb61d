// kspn_bench: the bench_kaspan command line (tool/bench_kaspan/src/main.cpp)
// on one B200, writing the same statistic JSON
// (kaspan/debug/statistic.hpp:123-205) so the reference's plotting scripts
// read its runs.
//
//   kspn_bench (--kagen_option_string <s> | --manifest_file <f>) --output_file <f>
//              [--variant (hpc_like | hpc_trim_ex | ispan_like | trim_ex |
//                          trim_ex_light_residual | trim_ex_residual | fast)]
//              [--repeat <k>]
//
// Graphs: a manifest (kspn_manifest_read / kspn_manifest_load), or a subset
// of KaGen option strings generated on the device with the library's seeded
// generators (KaGen itself is not linked): "gnm-directed;n=..;m=..;seed=..",
// "rmat;directed;n=..;m=..;a=..;b=..;c=..;seed=.." (n a power of two) and
// "rgg2d;n=..;avg_degree=..;seed=..".  Without --variant the reference's
// default phase order runs (KSPN_PIPELINE_REFERENCE, as bench_kaspan's
// `scc`); "fast" selects the library's own pipeline.
//
// JSON: {"0":{"benchmark":{"duration":ns, "memory", "world_rank", "world_size",
// "memcheck", "callgrind", "load"|"kagen":{"duration"}, "n", "local_n", "m",
// "local_fw_m", "local_bw_m", "scc":{"duration", one object per phase that
// ran: "trim_1_first", "forward_backward_search", "trim_1_normal", "trim",
// "trim_2", "residual", "color", "normalise", each with "duration" (device
// ns) and "decided_count"}, "local_component_count",
// "global_component_count"}}}.  With --repeat k the last of k runs is
// reported (the first ones warm the context).
#include "kspn.h"

#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace {

[[noreturn]] void
usage(char const* argv0)
{
  std::fprintf(stderr,
               "usage: %s (--kagen_option_string <kagen_option_string> | --manifest_file <manifest_file>) --output_file <output_file> "
               "[--variant (hpc_like | hpc_trim_ex | ispan_like | trim_ex | trim_ex_light_residual | trim_ex_residual | fast)] [--repeat <k>]\n",
               argv0);
  std::exit(1);
}

[[noreturn]] void
die(char const* what, int rc, kspn_context* ctx)
{
  std::fprintf(stderr, "kspn_bench: %s: %s (%s)\n", what, kspn_strerror(rc), ctx ? kspn_last_error(ctx) : "");
  std::exit(2);
}

#define CHECK(call, what)                  \
  do {                                     \
    int const rc_ = (call);                \
    if (rc_ != KSPN_OK) die(what, rc_, ctx); \
  } while (0)

uint64_t
now_ns()
{
  return static_cast<uint64_t>(std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch()).count());
}

uint64_t
resident_bytes()
{
  std::ifstream in("/proc/self/statm");
  uint64_t      pages = 0, rss = 0;
  in >> pages >> rss;
  return rss * 4096;
}

std::map<std::string, std::string>
parse_kagen(std::string const& s, std::string& kind)
{
  std::map<std::string, std::string> kv;
  std::stringstream                  ss(s);
  std::string                        tok;
  bool                               first = true;
  while (std::getline(ss, tok, ';')) {
    if (first) {
      kind  = tok;
      first = false;
      continue;
    }
    size_t const eq = tok.find('=');
    if (eq == std::string::npos) kv[tok] = "";
    else kv[tok.substr(0, eq)] = tok.substr(eq + 1);
  }
  return kv;
}

struct device_graph
{
  uint32_t  n = 0;
  uint64_t  m = 0;
  uint64_t* fh = nullptr;
  uint32_t* fc = nullptr;
  uint64_t* bh = nullptr;
  uint32_t* bc = nullptr;
};

void*
dalloc(size_t bytes)
{
  void* p = nullptr;
  if (cudaMalloc(&p, bytes ? bytes : 4) != cudaSuccess) {
    std::fprintf(stderr, "kspn_bench: cudaMalloc of %zu bytes failed\n", bytes);
    std::exit(2);
  }
  return p;
}

device_graph
from_edges(kspn_context* ctx, uint32_t n, uint64_t draws, uint32_t* src, uint32_t* dst)
{
  device_graph g;
  g.n  = n;
  g.fh = static_cast<uint64_t*>(dalloc((static_cast<size_t>(n) + 1) * 8));
  g.fc = static_cast<uint32_t*>(dalloc(draws * 4));
  CHECK(kspn_build_csr(ctx, n, draws, src, dst, g.fh, g.fc, &g.m), "build_csr");
  g.bh = static_cast<uint64_t*>(dalloc((static_cast<size_t>(n) + 1) * 8));
  g.bc = static_cast<uint32_t*>(dalloc(g.m * 4));
  CHECK(kspn_transpose(ctx, n, g.m, g.fh, g.fc, g.bh, g.bc), "transpose");
  return g;
}

device_graph
generate(kspn_context* ctx, std::string const& option)
{
  std::string kind;
  auto        kv  = parse_kagen(option, kind);
  auto        num = [&](char const* k, double dflt) { return kv.count(k) ? std::strtod(kv[k].c_str(), nullptr) : dflt; };
  uint64_t const seed = static_cast<uint64_t>(num("seed", 1));
  uint64_t const n    = static_cast<uint64_t>(num("n", 0));
  if (n == 0 || n >= 0xFFFFFFFFull) {
    std::fprintf(stderr, "kspn_bench: n must be in [1, 2^32 - 1)\n");
    std::exit(1);
  }
  if (kind == "gnm-directed" || kind == "rmat") {
    uint64_t const draws = static_cast<uint64_t>(num("m", 0));
    auto*          src   = static_cast<uint32_t*>(dalloc(draws * 4));
    auto*          dst   = static_cast<uint32_t*>(dalloc(draws * 4));
    if (kind == "gnm-directed") CHECK(kspn_gen_gnm(ctx, static_cast<uint32_t>(n), draws, seed, src, dst), "gen_gnm");
    else {
      int const scale = static_cast<int>(std::lround(std::log2(static_cast<double>(n))));
      if ((1ull << scale) != n) {
        std::fprintf(stderr, "kspn_bench: rmat needs n a power of two\n");
        std::exit(1);
      }
      double const   a = num("a", 0.57), b = num("b", 0.19), c = num("c", 0.19);
      double const   s = 4294967296.0;
      uint64_t const ta = static_cast<uint64_t>(std::floor(a * s)), tab = static_cast<uint64_t>(std::floor((a + b) * s)), tabc = static_cast<uint64_t>(std::floor((a + b + c) * s));
      CHECK(kspn_gen_rmat(ctx, scale, draws, seed, ta, tab, tabc, 1, src, dst), "gen_rmat");
    }
    device_graph g = from_edges(ctx, static_cast<uint32_t>(n), draws, src, dst);
    cudaFree(src);
    cudaFree(dst);
    return g;
  }
  if (kind == "rgg2d") {
    double const   deg = num("avg_degree", 8.0);
    double const   r   = std::sqrt(deg / (3.14159265358979323846 * static_cast<double>(n)));
    uint32_t const gsz = static_cast<uint32_t>(std::max(1.0, std::floor(1.0 / r)));
    uint64_t const r2  = static_cast<uint64_t>(std::floor(r * r * 1152921504606846976.0)); // 2^60
    uint64_t       m   = 0;
    CHECK(kspn_gen_rgg(ctx, static_cast<uint32_t>(n), seed, gsz, r2, nullptr, nullptr, 0, &m), "gen_rgg");
    auto* src = static_cast<uint32_t*>(dalloc(m * 4));
    auto* dst = static_cast<uint32_t*>(dalloc(m * 4));
    CHECK(kspn_gen_rgg(ctx, static_cast<uint32_t>(n), seed, gsz, r2, src, dst, m, &m), "gen_rgg");
    device_graph g = from_edges(ctx, static_cast<uint32_t>(n), m, src, dst);
    cudaFree(src);
    cudaFree(dst);
    return g;
  }
  std::fprintf(stderr, "kspn_bench: unsupported generator \"%s\" (gnm-directed, rmat, rgg2d)\n", kind.c_str());
  std::exit(1);
}

} // namespace

int
main(int argc, char** argv)
{
  char const* kagen = nullptr;
  char const* mfile = nullptr;
  char const* out   = nullptr;
  char const* var   = nullptr;
  int         reps  = 1;
  for (int i = 1; i < argc; ++i) {
    auto next = [&]() -> char const* {
      if (i + 1 >= argc) usage(argv[0]);
      return argv[++i];
    };
    if (!std::strcmp(argv[i], "--kagen_option_string")) kagen = next();
    else if (!std::strcmp(argv[i], "--manifest_file")) mfile = next();
    else if (!std::strcmp(argv[i], "--output_file")) out = next();
    else if (!std::strcmp(argv[i], "--variant")) var = next();
    else if (!std::strcmp(argv[i], "--repeat")) reps = std::max(1, std::atoi(next()));
    else usage(argv[0]);
  }
  if ((kagen == nullptr) == (mfile == nullptr) || out == nullptr) usage(argv[0]);

  kspn_options opt;
  kspn_options_default(&opt);
  opt.pipeline = KSPN_PIPELINE_REFERENCE;
  if (var) {
    static std::map<std::string, int> const variants{ { "hpc_like", KSPN_PIPELINE_HPC_LIKE },
                                                      { "hpc_trim_ex", KSPN_PIPELINE_HPC_TRIM_EX },
                                                      { "ispan_like", KSPN_PIPELINE_ISPAN_LIKE },
                                                      { "trim_ex", KSPN_PIPELINE_TRIM_EX },
                                                      { "trim_ex_light_residual", KSPN_PIPELINE_TRIM_EX_LIGHT_RESIDUAL },
                                                      { "trim_ex_residual", KSPN_PIPELINE_TRIM_EX_RESIDUAL },
                                                      { "fast", KSPN_PIPELINE_FAST } };
    auto const it = variants.find(var);
    if (it == variants.end()) usage(argv[0]);
    opt.pipeline = it->second;
  }

  uint64_t const t_bench = now_ns();
  kspn_context*  ctx     = nullptr;
  CHECK(kspn_context_create(0, &ctx), "context");

  uint64_t const t_load = now_ns();
  device_graph   g;
  if (mfile) {
    kspn_manifest mf;
    CHECK(kspn_manifest_read(mfile, &mf), "manifest_read");
    if (mf.node_count >= 0xFFFFFFFFull) die("manifest: node_count too large", KSPN_ERR_INVALID_ARGUMENT, ctx);
    g.n  = static_cast<uint32_t>(mf.node_count);
    g.m  = mf.edge_count;
    g.fh = static_cast<uint64_t*>(dalloc((static_cast<size_t>(g.n) + 1) * 8));
    g.bh = static_cast<uint64_t*>(dalloc((static_cast<size_t>(g.n) + 1) * 8));
    g.fc = static_cast<uint32_t*>(dalloc(g.m * 4));
    g.bc = static_cast<uint32_t*>(dalloc(g.m * 4));
    CHECK(kspn_manifest_load(ctx, &mf, g.fh, g.fc, g.bh, g.bc), "manifest_load");
  } else g = generate(ctx, kagen);
  cudaDeviceSynchronize();
  uint64_t const load_ns = now_ns() - t_load;

  auto*      d_ids = static_cast<uint32_t*>(dalloc(static_cast<size_t>(g.n) * 4));
  kspn_stats st;
  uint64_t   scc_ns = 0;
  for (int r = 0; r < reps; ++r) {
    uint64_t const t0 = now_ns();
    CHECK(kspn_scc_device(ctx, g.n, g.m, g.fh, g.fc, g.bh, g.bc, d_ids, &opt, &st), "scc");
    scc_ns = now_ns() - t0;
  }
  std::vector<uint32_t> ids(g.n);
  cudaMemcpy(ids.data(), d_ids, static_cast<size_t>(g.n) * 4, cudaMemcpyDeviceToHost);
  uint64_t comps = 0;
  for (uint32_t v = 0; v < g.n; ++v) comps += ids[v] == v;
  uint64_t const bench_ns = now_ns() - t_bench;

  // the statistic JSON (one rank)
  static char const* const phase_name[KSPN_PHASES] = { "trim_1_first", "trim", "forward_backward_search", "trim_1_normal", "color", "trim_2", "residual", "normalise" };
  static int const         order[KSPN_PHASES]      = { KSPN_PHASE_TRIM_FIRST, KSPN_PHASE_FWBW, KSPN_PHASE_TRIM_NORMAL, KSPN_PHASE_TRIM, KSPN_PHASE_TRIM2, KSPN_PHASE_RESIDUAL, KSPN_PHASE_LABEL, KSPN_PHASE_CANON };
  std::ostringstream       js;
  js << "{\"0\":{\"benchmark\":{\"duration\":" << bench_ns << ",\"memory\":" << resident_bytes() << ",\"world_rank\":0,\"world_size\":1,\"memcheck\":0,\"callgrind\":0";
  js << ",\"" << (mfile ? "load" : "kagen") << "\":{\"duration\":" << load_ns << "}";
  js << ",\"n\":" << g.n << ",\"local_n\":" << g.n << ",\"m\":" << g.m << ",\"local_fw_m\":" << g.m << ",\"local_bw_m\":" << g.m;
  js << ",\"scc\":{\"duration\":" << scc_ns;
  for (int k : order) {
    if (st.decided[k] == 0 && st.ms[k] <= 0.0) continue;
    js << ",\"" << phase_name[k] << "\":{\"duration\":" << static_cast<uint64_t>(st.ms[k] * 1e6) << ",\"decided_count\":" << st.decided[k] << "}";
  }
  js << ",\"device_duration\":" << static_cast<uint64_t>(st.ms_total * 1e6) << ",\"edges_scanned\":" << st.edges_scanned << "}";
  js << ",\"local_component_count\":" << comps << ",\"global_component_count\":" << comps << "}}}";
  std::ofstream f(out);
  f << js.str() << "\n";
  if (!f.good()) {
    std::fprintf(stderr, "kspn_bench: cannot write %s\n", out);
    return 2;
  }
  std::printf("n=%u m=%llu components=%llu scc=%.3f ms (device %.3f ms)\n", g.n, static_cast<unsigned long long>(g.m), static_cast<unsigned long long>(comps), scc_ns * 1e-6, st.ms_total);
  kspn_context_destroy(ctx);
  return 0;
}
