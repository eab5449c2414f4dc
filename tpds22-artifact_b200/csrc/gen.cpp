// Synthetic inputs (host, C++): seeded uniform arrays, R-MAT and 2-D grid
// graphs in CSR form, symmetric edge weights, and the Galois/Lonestar `.gr` v1
// binary graph format.
//
// The reference reads graphs only from `.gr` files (CSRGraph::readFromGR,
// LONESTAR/rt/src/csr_graph.cu:152-237) produced by downloads that are not
// available here; these generators produce the stand-in inputs in the same
// layout (CSRGraph: row_start[n+1], edge_dst[m], edge_data[m] as 32-bit
// values, LONESTAR/rt/include/csr_graph.h.prehip:20-103).
//
// Random numbers: splitmix64 (Steele, Lea, Flood 2014) seeds xoshiro256**
// (Blackman, Vigna 2018); both are published algorithms restated here.  Work
// is split into fixed-size blocks with one stream per block, so results do not
// depend on the number of host threads.
// R-MAT: Chakrabarti, Zhan, Faloutsos, "R-MAT: A Recursive Model for Graph
// Mining", SDM 2004: each edge descends `scale` levels choosing a quadrant with
// probabilities a, b, c, d = 1-a-b-c.
#include "gsrb.h"
#include <stdint.h>
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

namespace {

inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}
inline uint64_t mix64(uint64_t x) {
  uint64_t s = x;
  return splitmix64(s);
}
inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

struct Xoshiro {
  uint64_t s[4];
  explicit Xoshiro(uint64_t seed) {
    uint64_t t = seed;
    for (auto& w : s) w = splitmix64(t);
  }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

uint64_t block_seed(uint64_t seed, uint64_t block) { return mix64(seed ^ mix64(block + 0x5851f42d4c957f2dull)); }

template <class F>
void parallel_blocks(uint64_t nblocks, F f) {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  if (nt > nblocks) nt = (unsigned)(nblocks ? nblocks : 1);
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> th;
  for (unsigned t = 0; t < nt; ++t)
    th.emplace_back([&]() {
      for (;;) {
        uint64_t b = next.fetch_add(1);
        if (b >= nblocks) break;
        f(b);
      }
    });
  for (auto& t : th) t.join();
}

constexpr uint64_t kBlock = 1ull << 16;

}  // namespace

extern "C" uint32_t gsrb_edge_weight(uint32_t u, uint32_t v, uint64_t seed, int32_t lo, int32_t hi) {
  const uint32_t a = u < v ? u : v, b = u < v ? v : u;
  const uint64_t h = mix64(seed ^ (((uint64_t)a << 32) | b));
  return (uint32_t)(lo + (int32_t)(h % (uint64_t)(hi - lo + 1)));
}

extern "C" {

gsrb_status_t gsrb_gen_uniform_i32(uint64_t seed, size_t n, int32_t lo, int32_t hi, int32_t* out) {
  if ((n && !out) || hi < lo) return GSRB_ERR_ARG;
  const uint64_t span = (uint64_t)((int64_t)hi - (int64_t)lo) + 1;
  parallel_blocks((n + kBlock - 1) / kBlock, [&](uint64_t b) {
    Xoshiro r(block_seed(seed, b));
    const uint64_t e = std::min<uint64_t>(n, (b + 1) * kBlock);
    for (uint64_t i = b * kBlock; i < e; ++i) out[i] = (int32_t)((int64_t)lo + (int64_t)(r.next() % span));
  });
  return GSRB_OK;
}

gsrb_status_t gsrb_gen_uniform_f32(uint64_t seed, size_t n, float* out) {
  if (n && !out) return GSRB_ERR_ARG;
  parallel_blocks((n + kBlock - 1) / kBlock, [&](uint64_t b) {
    Xoshiro r(block_seed(seed, b));
    const uint64_t e = std::min<uint64_t>(n, (b + 1) * kBlock);
    for (uint64_t i = b * kBlock; i < e; ++i) out[i] = (float)(r.next() >> 40) * (1.0f / 16777216.0f);
  });
  return GSRB_OK;
}

void gsrb_host_csr_free(gsrb_host_csr_t* g) {
  if (!g) return;
  free(g->row_start);
  free(g->edge_dst);
  free(g->edge_data);
  memset(g, 0, sizeof(*g));
}

// Build a symmetric, self-loop-free, duplicate-free CSR with sorted rows from a
// directed edge list (both directions are inserted).
gsrb_status_t gsrb_csr_from_edges(uint32_t n, uint64_t m, const uint32_t* src, const uint32_t* dst,
                                  int symmetrize, uint64_t weight_seed, int32_t wlo, int32_t whi,
                                  gsrb_host_csr_t* out) {
  if (!out || (m && (!src || !dst))) return GSRB_ERR_ARG;
  memset(out, 0, sizeof(*out));
  std::vector<std::atomic<uint32_t>> deg(n);
  for (auto& d : deg) d.store(0, std::memory_order_relaxed);
  const uint64_t nb = (m + kBlock - 1) / kBlock;
  parallel_blocks(nb, [&](uint64_t b) {
    const uint64_t e = std::min<uint64_t>(m, (b + 1) * kBlock);
    for (uint64_t i = b * kBlock; i < e; ++i) {
      if (src[i] == dst[i] || src[i] >= n || dst[i] >= n) continue;
      deg[src[i]].fetch_add(1, std::memory_order_relaxed);
      if (symmetrize) deg[dst[i]].fetch_add(1, std::memory_order_relaxed);
    }
  });
  std::vector<uint64_t> off(n + 1, 0);
  for (uint32_t v = 0; v < n; ++v) off[v + 1] = off[v] + deg[v].load(std::memory_order_relaxed);
  const uint64_t total = off[n];
  uint32_t* adj = (uint32_t*)malloc(sizeof(uint32_t) * (total ? total : 1));
  if (!adj) return GSRB_ERR_NOMEM;
  std::vector<std::atomic<uint64_t>> pos(n);
  for (uint32_t v = 0; v < n; ++v) pos[v].store(off[v], std::memory_order_relaxed);
  parallel_blocks(nb, [&](uint64_t b) {
    const uint64_t e = std::min<uint64_t>(m, (b + 1) * kBlock);
    for (uint64_t i = b * kBlock; i < e; ++i) {
      const uint32_t u = src[i], v = dst[i];
      if (u == v || u >= n || v >= n) continue;
      adj[pos[u].fetch_add(1, std::memory_order_relaxed)] = v;
      if (symmetrize) adj[pos[v].fetch_add(1, std::memory_order_relaxed)] = u;
    }
  });
  // sort + dedup every row (row order makes the result independent of threads)
  std::vector<uint32_t> newdeg(n, 0);
  const uint64_t vb = (n + 4095) / 4096;
  parallel_blocks(vb, [&](uint64_t b) {
    const uint32_t e = (uint32_t)std::min<uint64_t>(n, (b + 1) * 4096);
    for (uint32_t v = (uint32_t)(b * 4096); v < e; ++v) {
      uint32_t* r0 = adj + off[v];
      uint32_t* r1 = adj + off[v + 1];
      std::sort(r0, r1);
      newdeg[v] = (uint32_t)(std::unique(r0, r1) - r0);
    }
  });
  uint64_t mm = 0;
  for (uint32_t v = 0; v < n; ++v) mm += newdeg[v];
  if (mm >= (1ull << 32)) { free(adj); return GSRB_ERR_OVERFLOW; }
  out->nnodes = n;
  out->nedges = mm;
  out->row_start = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
  out->edge_dst = (uint32_t*)malloc(sizeof(uint32_t) * (mm ? mm : 1));
  out->edge_data = (int32_t*)malloc(sizeof(int32_t) * (mm ? mm : 1));
  if (!out->row_start || !out->edge_dst || !out->edge_data) {
    free(adj);
    gsrb_host_csr_free(out);
    return GSRB_ERR_NOMEM;
  }
  out->row_start[0] = 0;
  for (uint32_t v = 0; v < n; ++v) out->row_start[v + 1] = out->row_start[v] + newdeg[v];
  parallel_blocks(vb, [&](uint64_t b) {
    const uint32_t e = (uint32_t)std::min<uint64_t>(n, (b + 1) * 4096);
    for (uint32_t v = (uint32_t)(b * 4096); v < e; ++v) {
      const uint32_t d = newdeg[v];
      const uint32_t base = out->row_start[v];
      memcpy(out->edge_dst + base, adj + off[v], sizeof(uint32_t) * d);
      for (uint32_t j = 0; j < d; ++j)
        out->edge_data[base + j] = (int32_t)gsrb_edge_weight(v, out->edge_dst[base + j], weight_seed, wlo, whi);
    }
  });
  free(adj);
  return GSRB_OK;
}

gsrb_status_t gsrb_gen_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c, uint64_t seed,
                            int32_t wlo, int32_t whi, gsrb_host_csr_t* out) {
  if (!out || scale < 1 || scale > 30 || edgefactor < 1 || a < 0 || b < 0 || c < 0 || a + b + c > 1.0 ||
      whi < wlo)
    return GSRB_ERR_ARG;
  const uint32_t n = 1u << scale;
  const uint64_t m = (uint64_t)edgefactor << scale;
  std::vector<uint32_t> src(m), dst(m);
  const double ab = a + b, abc = a + b + c;
  parallel_blocks((m + kBlock - 1) / kBlock, [&](uint64_t blk) {
    Xoshiro r(block_seed(seed, blk));
    const uint64_t e = std::min<uint64_t>(m, (blk + 1) * kBlock);
    for (uint64_t i = blk * kBlock; i < e; ++i) {
      uint32_t u = 0, v = 0;
      for (int l = 0; l < scale; ++l) {
        const double x = r.uniform();
        const uint32_t bu = x >= ab ? 1u : 0u;                       // quadrants c, d
        const uint32_t bv = (x >= a && x < ab) || x >= abc ? 1u : 0u;  // quadrants b, d
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      src[i] = u;
      dst[i] = v;
    }
  });
  return gsrb_csr_from_edges(n, m, src.data(), dst.data(), 1, seed ^ 0xC0FFEEull, wlo, whi, out);
}

gsrb_status_t gsrb_gen_grid2d(int32_t width, int32_t height, uint64_t seed, int32_t wlo, int32_t whi,
                              gsrb_host_csr_t* out) {
  if (!out || width < 1 || height < 1 || whi < wlo) return GSRB_ERR_ARG;
  const uint64_t n64 = (uint64_t)width * height;
  if (n64 >= (1ull << 31)) return GSRB_ERR_ARG;
  const uint32_t n = (uint32_t)n64, W = (uint32_t)width, H = (uint32_t)height;
  memset(out, 0, sizeof(*out));
  const uint64_t m = 2ull * ((uint64_t)(W - 1) * H + (uint64_t)W * (H - 1));
  out->nnodes = n;
  out->nedges = m;
  out->row_start = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
  out->edge_dst = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  out->edge_data = (int32_t*)malloc(sizeof(int32_t) * (m ? m : 1));
  if (!out->row_start || !out->edge_dst || !out->edge_data) {
    gsrb_host_csr_free(out);
    return GSRB_ERR_NOMEM;
  }
  uint32_t e = 0;
  for (uint32_t v = 0; v < n; ++v) {
    out->row_start[v] = e;
    const uint32_t r = v / W, col = v % W;
    // neighbours in increasing id order: up, left, right, down
    if (r > 0) out->edge_dst[e++] = v - W;
    if (col > 0) out->edge_dst[e++] = v - 1;
    if (col + 1 < W) out->edge_dst[e++] = v + 1;
    if (r + 1 < H) out->edge_dst[e++] = v + W;
  }
  out->row_start[n] = e;
  const uint64_t wseed = seed ^ 0xC0FFEEull;
  parallel_blocks(((uint64_t)n + 65535) / 65536, [&](uint64_t b) {
    const uint32_t hi = (uint32_t)std::min<uint64_t>(n, (b + 1) * 65536);
    for (uint32_t v = (uint32_t)(b * 65536); v < hi; ++v)
      for (uint32_t j = out->row_start[v]; j < out->row_start[v + 1]; ++j)
        out->edge_data[j] = (int32_t)gsrb_edge_weight(v, out->edge_dst[j], wseed, wlo, whi);
  });
  return GSRB_OK;
}

// `.gr` v1: u64 version(=1), u64 sizeEdgeTy, u64 numNodes, u64 numEdges,
// u64 outIdx[numNodes] (row END offsets), u32 dst[numEdges], one u32 of padding
// when numEdges is odd, then numEdges edge values of sizeEdgeTy bytes.
// (LONESTAR/rt/src/csr_graph.cu:183-226; little-endian host assumed, as there.)
gsrb_status_t gsrb_gr_write(const char* path, const gsrb_host_csr_t* g, int32_t with_weights) {
  if (!path || !g || !g->row_start || (g->nedges && !g->edge_dst)) return GSRB_ERR_ARG;
  FILE* f = fopen(path, "wb");
  if (!f) return GSRB_ERR_ARG;
  const uint64_t hdr[4] = {1, with_weights ? 4u : 0u, g->nnodes, g->nedges};
  bool ok = fwrite(hdr, sizeof(hdr), 1, f) == 1;
  std::vector<uint64_t> outIdx(g->nnodes);
  for (uint32_t v = 0; v < g->nnodes; ++v) outIdx[v] = g->row_start[v + 1];
  if (g->nnodes) ok = ok && fwrite(outIdx.data(), sizeof(uint64_t), g->nnodes, f) == g->nnodes;
  if (g->nedges) ok = ok && fwrite(g->edge_dst, sizeof(uint32_t), g->nedges, f) == g->nedges;
  if (g->nedges & 1) {
    const uint32_t pad = 0;
    ok = ok && fwrite(&pad, sizeof(pad), 1, f) == 1;
  }
  if (with_weights && g->nedges) {
    if (!g->edge_data) ok = false;
    else ok = ok && fwrite(g->edge_data, sizeof(int32_t), g->nedges, f) == g->nedges;
  }
  ok = (fclose(f) == 0) && ok;
  return ok ? GSRB_OK : GSRB_ERR_ARG;
}

gsrb_status_t gsrb_gr_read(const char* path, gsrb_host_csr_t* out) {
  if (!path || !out) return GSRB_ERR_ARG;
  memset(out, 0, sizeof(*out));
  FILE* f = fopen(path, "rb");
  if (!f) return GSRB_ERR_ARG;
  uint64_t hdr[4];
  if (fread(hdr, sizeof(hdr), 1, f) != 1 || hdr[0] != 1 || (hdr[1] != 0 && hdr[1] != 4) ||
      hdr[2] >= (1ull << 32) || hdr[3] >= (1ull << 32)) {
    fclose(f);
    return GSRB_ERR_ARG;
  }
  const uint32_t n = (uint32_t)hdr[2];
  const uint64_t m = hdr[3];
  out->nnodes = n;
  out->nedges = m;
  out->row_start = (uint32_t*)malloc(sizeof(uint32_t) * ((size_t)n + 1));
  out->edge_dst = (uint32_t*)malloc(sizeof(uint32_t) * (m ? m : 1));
  out->edge_data = (int32_t*)calloc(m ? m : 1, sizeof(int32_t));
  std::vector<uint64_t> outIdx(n);
  bool ok = out->row_start && out->edge_dst && out->edge_data;
  if (ok && n) ok = fread(outIdx.data(), sizeof(uint64_t), n, f) == n;
  if (ok && m) ok = fread(out->edge_dst, sizeof(uint32_t), m, f) == m;
  if (ok && (m & 1)) {
    uint32_t pad;
    ok = fread(&pad, sizeof(pad), 1, f) == 1;
  }
  if (ok && hdr[1] == 4 && m) ok = fread(out->edge_data, sizeof(int32_t), m, f) == m;
  fclose(f);
  if (ok) {
    out->row_start[0] = 0;
    for (uint32_t v = 0; v < n; ++v) {
      if (outIdx[v] < (v ? outIdx[v - 1] : 0) || outIdx[v] > m) { ok = false; break; }
      out->row_start[v + 1] = (uint32_t)outIdx[v];
    }
    if (ok && n && out->row_start[n] != m) ok = false;
    for (uint64_t j = 0; ok && j < m; ++j)
      if (out->edge_dst[j] >= n) ok = false;
  }
  if (!ok) {
    gsrb_host_csr_free(out);
    return GSRB_ERR_ARG;
  }
  return GSRB_OK;
}

}  // extern "C"
