// Grouped persistent FP64 DMMA GEMM and its autotuner.
//
// A launch covers the tiles of many independent products of different shapes: the problems'
// descriptors sit in a device table with the prefix sums of their tile counts, and a persistent grid
// (SMs x resident CTAs) walks the concatenated tile list with a fixed stride, each CTA finding its
// problem by binary search and running the same tile body as the one-problem kernel (gemm_tile.cuh).
// Split-K partials and the mirrored lower triangles of Hermitian outputs are finished by one grouped
// launch each.  The tile configuration and split count of every problem come from the autotuner, per
// problem shape, so a problem's arithmetic (and its rounding) is the same in any group.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <unordered_map>

#include "gemm_tile.cuh"
#include "grouped.cuh"

namespace rr {

int64_t launches();  // kernels launched by the library so far (ri_core.cu)

namespace {

using namespace gk;

struct GroupArgs {
  const Params* probs;
  const int64_t* off;  // off[i]: first tile (or element) of problem i; ascending
  int n;
  int64_t total;
};

__device__ __forceinline__ int find_problem(const int64_t* off, int n, int64_t t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX, int V>
__global__ void __launch_bounds__(32 * WM * WN) dgemm_grouped_kernel(const GroupArgs g) {
  using CF = Cfg<MT, NT, WM, WN, AK, BKM, CPLX>;
  extern __shared__ __align__(16) double smem[];
  __shared__ Params sp;
  for (int64_t t = blockIdx.x; t < g.total; t += gridDim.x) {
    const int pi = find_problem(g.off, g.n, t);
    __syncthreads();  // the previous tile is done with sp and the ring
    if (threadIdx.x == 0) sp = g.probs[pi];
    __syncthreads();
    const int64_t lt = t - g.off[pi];
    const int64_t tx = (sp.N + CF::BN - 1) / CF::BN, ty = (sp.M + CF::BM - 1) / CF::BM;
    const int64_t bz = lt / (tx * ty), rem = lt % (tx * ty);
    const int64_t m0 = (rem / tx) * CF::BM, n0 = (rem % tx) * CF::BN;
    if (sp.upper_only && m0 > n0 + CF::BN - 1) continue;
    dgemm_tile<MT, NT, WM, WN, AK, BKM, CPLX, V, false>(sp, n0, m0, bz, smem, 0);
  }
}

template <int PL>
__global__ void splitk_reduce_grouped_kernel(const GroupArgs g) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < g.total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int pi = find_problem(g.off, g.n, idx);
    splitk_reduce_elem<PL>(g.probs[pi], idx - g.off[pi]);
  }
}

template <int PL>
__global__ void mirror_grouped_kernel(const GroupArgs g) {
  for (int64_t idx = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; idx < g.total;
       idx += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int pi = find_problem(g.off, g.n, idx);
    const Params& p = g.probs[pi];
    mirror_elem<PL>(p.C, p.M, p.ldc, p.strideC, p.mirror, idx - g.off[pi]);
  }
}

// Tile configurations: real 0 32x32, 1 64x64, 2 80x80, 3 8x128, 4 16x128, 5 32x128, 6 40x80;
// complex 0 32x32, 1 32x64.
struct TileDims {
  int bm, bn;
};
constexpr TileDims kReal[7] = {{32, 32}, {64, 64}, {80, 80}, {8, 128}, {16, 128}, {32, 128}, {40, 80}};
constexpr TileDims kCplx[2] = {{32, 32}, {32, 64}};
TileDims dims_of(bool cplx, int cfg) { return cplx ? kCplx[cfg] : kReal[cfg]; }

template <int MT, int NT, int WM, int WN, bool AK, bool BKM, bool CPLX, int V = 1>
void launch_grouped(const GroupArgs& g, cudaStream_t s) {
  using CF = Cfg<MT, NT, WM, WN, AK, BKM, CPLX>;
  auto kern = dgemm_grouped_kernel<MT, NT, WM, WN, AK, BKM, CPLX, V>;
  static std::atomic<bool> attr[kMaxDevices];
  static int occ[kMaxDevices];
  const int dev = current_device();
  once_per_device(attr, [&] {
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, CF::SMEM_BYTES));
    RR_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
    int o = 0;
    RR_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kern, CF::THREADS, CF::SMEM_BYTES));
    occ[dev] = std::max(o, 1);
  });
  const int64_t grid = std::min<int64_t>(g.total, static_cast<int64_t>(sm_count_current()) * occ[dev]);
  kern<<<static_cast<unsigned>(std::max<int64_t>(grid, 1)), CF::THREADS, CF::SMEM_BYTES, s>>>(g);
  RR_LAUNCH_CHECK();
}

template <bool AK, bool BKM, int V>
void launch_real_cfg_v(int cfg, const GroupArgs& g, cudaStream_t s) {
  switch (cfg) {
    case 0: return launch_grouped<2, 2, 2, 2, AK, BKM, false, V>(g, s);
    case 1: return launch_grouped<4, 4, 2, 2, AK, BKM, false, V>(g, s);
    case 2: return launch_grouped<5, 5, 2, 2, AK, BKM, false, V>(g, s);
    case 3: return launch_grouped<1, 4, 1, 4, AK, BKM, false, V>(g, s);
    case 4: return launch_grouped<2, 4, 1, 4, AK, BKM, false, V>(g, s);
    case 5: return launch_grouped<4, 4, 1, 4, AK, BKM, false, V>(g, s);
    default: return launch_grouped<5, 2, 1, 5, AK, BKM, false, V>(g, s);
  }
}

template <bool AK, bool BKM>
void launch_real_cfg(int cfg, bool vec2, const GroupArgs& g, cudaStream_t s) {
  if (vec2) launch_real_cfg_v<AK, BKM, 2>(cfg, g, s);
  else launch_real_cfg_v<AK, BKM, 1>(cfg, g, s);
}

template <bool AK, bool BKM>
void launch_cplx_cfg(int cfg, const GroupArgs& g, cudaStream_t s) {
  if (cfg == 0) launch_grouped<2, 2, 2, 2, AK, BKM, true>(g, s);
  else launch_grouped<2, 4, 2, 2, AK, BKM, true>(g, s);
}

void launch_cfg(bool cplx, bool AK, bool BKM, int cfg, bool vec2, const GroupArgs& g, cudaStream_t s) {
  if (cplx) {
    if (AK && BKM) launch_cplx_cfg<true, true>(cfg, g, s);
    else if (AK) launch_cplx_cfg<true, false>(cfg, g, s);
    else if (BKM) launch_cplx_cfg<false, true>(cfg, g, s);
    else launch_cplx_cfg<false, false>(cfg, g, s);
  } else {
    if (AK && BKM) launch_real_cfg<true, true>(cfg, vec2, g, s);
    else if (AK) launch_real_cfg<true, false>(cfg, vec2, g, s);
    else if (BKM) launch_real_cfg<false, true>(cfg, vec2, g, s);
    else launch_real_cfg<false, false>(cfg, vec2, g, s);
  }
}

// 16-byte loads (real products only): 16-byte aligned bases and batch strides, even leading dims, even
// contiguous extents and an even k chunk, so that a pair of doubles never straddles a row end.
bool vec2_ok(const GemmDesc& d, int64_t kchunk) {
  if (d.cplx) return false;
  auto al = [](const void* q) { return (reinterpret_cast<uintptr_t>(q) & 15) == 0; };
  const bool AK = d.opA == Op::N, BKM = d.opB == Op::T;
  const bool a = al(d.A) && d.lda % 2 == 0 && d.strideA % 2 == 0 && (AK ? d.K % 2 == 0 : d.M % 2 == 0);
  const bool b = al(d.B) && d.ldb % 2 == 0 && d.strideB % 2 == 0 && (BKM ? d.K % 2 == 0 : d.N % 2 == 0);
  return a && b && kchunk % 2 == 0;
}

void check_desc(const GemmDesc& d) {
  RR_REQUIRE(d.M >= 0 && d.N >= 0 && d.K >= 0 && d.batch >= 0, RR_ERR_ARG, "gemm_grouped: negative size");
  RR_REQUIRE(!d.mirror || d.M == d.N, RR_ERR_ARG, "gemm_grouped: mirror needs a square output");
  RR_REQUIRE(d.mirror >= -1 && d.mirror <= 2, RR_ERR_ARG, "gemm_grouped: mirror must be -1, 0, 1 or 2");
  RR_REQUIRE(!d.mirror || (d.c_plane_rows == 0 && d.c_col_stride == 1), RR_ERR_ARG,
             "gemm_grouped: mirror with planar or strided output");
  RR_REQUIRE(d.c_col_stride >= 1 && (d.c_col_stride == 1 || !d.cplx), RR_ERR_ARG, "gemm_grouped: bad output column stride");
  RR_REQUIRE(!d.edot_out, RR_ERR_ARG, "gemm_grouped: no epilogue dot");
}

// Builds the launches of descs[i] with choice[i] (the autotuner's, or a candidate it is timing).
void grouped_build(const std::vector<GemmDesc>& descs, const std::vector<GemmChoice>& choice, cudaStream_t s,
                   TableRing& ring, DevBuf<double>& work, GroupedPlan& plan) {
  plan.launches.clear();
  plan.side = &ring.side;
  struct Item {
    size_t i;
    int cfg, splits;
    int64_t kc, tiles, wneed;
  };
  std::vector<Item> items;
  items.reserve(descs.size());
  int64_t wtotal = 0;
  for (size_t i = 0; i < descs.size(); ++i) {
    const GemmDesc& d = descs[i];
    check_desc(d);
    if (d.M == 0 || d.N == 0 || d.batch == 0) continue;
    const TileDims td = dims_of(d.cplx, choice[i].cfg);
    int splits = d.K > 0 ? std::max(1, choice[i].splits) : 1;
    int64_t kc = round_up(std::max<int64_t>((d.K + splits - 1) / splits, 1), gk::KT);
    splits = d.K > 0 ? static_cast<int>((d.K + kc - 1) / kc) : 1;
    if (splits <= 1) { splits = 1; kc = std::max<int64_t>(d.K, 1); }
    const int64_t tiles = static_cast<int64_t>(ceil_div(d.M, td.bm)) * ceil_div(d.N, td.bn) * d.batch * splits;
    const int64_t wneed = splits > 1 ? d.batch * splits * d.M * d.N * (d.cplx ? 2 : 1) : 0;
    items.push_back({i, choice[i].cfg, splits, kc, tiles, wneed});
    wtotal += round_up(wneed, 32);
  }
  if (items.empty()) return;
  if (static_cast<int64_t>(work.n) < wtotal) {
    RR_CUDA(cudaStreamSynchronize(s));  // launches in flight may still read the old scratch
    work.alloc(static_cast<size_t>(wtotal));
  }
  std::vector<Params> prm(items.size());
  int64_t woff = 0;
  for (size_t k = 0; k < items.size(); ++k) {
    const GemmDesc& d = descs[items[k].i];
    Params& p = prm[k];
    p = Params{};
    p.M = d.M; p.N = d.N; p.K = d.K;
    p.A = d.A; p.lda = d.lda; p.strideA = d.strideA;
    p.B = d.B; p.ldb = d.ldb; p.strideB = d.strideB;
    p.C = d.C; p.ldc = d.ldc; p.strideC = d.strideC;
    p.alpha = d.alpha; p.beta = d.beta; p.batch = d.batch;
    p.splits = items[k].splits; p.kchunk = items[k].kc;
    p.work = items[k].wneed ? work.p + woff : nullptr;
    woff += round_up(items[k].wneed, 32);
    p.signA = d.conjA ? -1.0 : 1.0;
    p.signB = d.conjB ? -1.0 : 1.0;
    p.c_plane_rows = d.c_plane_rows; p.c_plane_stride = d.c_plane_stride;
    p.ccs = d.c_col_stride;
    p.upper_only = d.mirror != 0;
    p.mirror = d.mirror;
  }
  // one launch per (element kind, layout, configuration); inside it the longest-K problems first, so
  // the fixed-stride walk spreads them over the grid
  std::vector<std::pair<int, std::vector<size_t>>> groups;  // few keys: a sorted small vector
  for (size_t k = 0; k < items.size(); ++k) {
    const GemmDesc& d = descs[items[k].i];
    const int key = (vec2_ok(d, items[k].kc) ? 10000 : 0) + (d.cplx ? 1000 : 0) + (d.opA == Op::N ? 100 : 0) +
                    (d.opB == Op::T ? 10 : 0) + items[k].cfg;
    auto it = std::find_if(groups.begin(), groups.end(), [&](const auto& g) { return g.first == key; });
    if (it == groups.end()) {
      groups.emplace_back(key, std::vector<size_t>{});
      it = groups.end() - 1;
    }
    it->second.push_back(k);
  }
  std::sort(groups.begin(), groups.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
  for (auto& [key, ks] : groups) {
    std::stable_sort(ks.begin(), ks.end(), [&](size_t a, size_t b) {
      return prm[a].kchunk * prm[a].M > prm[b].kchunk * prm[b].M;
    });
    std::vector<Params> gp;
    std::vector<int64_t> off;
    int64_t total = 0;
    for (size_t k : ks) {
      gp.push_back(prm[k]);
      off.push_back(total);
      total += items[k].tiles;
    }
    GroupedLaunch L{};
    L.kind = 0;
    L.probs = ring.put(gp.data(), sizeof(Params) * gp.size(), s);
    L.off = static_cast<const int64_t*>(ring.put(off.data(), sizeof(int64_t) * off.size(), s));
    L.n = static_cast<int>(gp.size());
    L.total = total;
    L.vec2 = key >= 10000;
    L.cplx = (key / 1000) % 10 == 1;
    L.AK = (key / 100) % 10 == 1;
    L.BKM = (key / 10) % 10 == 1;
    L.cfg = key % 10;
    plan.launches.push_back(L);
  }
  // split-K reductions, then mirrors of the one-pass upper-only products (the reduction mirrors its own)
  for (int pl = 1; pl <= 2; ++pl)
    for (int pass = 0; pass < 2; ++pass) {
      std::vector<Params> gp;
      std::vector<int64_t> off;
      int64_t total = 0;
      for (size_t k = 0; k < items.size(); ++k) {
        const GemmDesc& d = descs[items[k].i];
        if ((d.cplx ? 2 : 1) != pl) continue;
        const bool take = pass == 0 ? items[k].splits > 1 : ((d.mirror == 1 || d.mirror == -1) && items[k].splits == 1);
        if (!take) continue;
        gp.push_back(prm[k]);
        off.push_back(total);
        total += d.batch * d.M * d.N;
      }
      if (gp.empty()) continue;
      GroupedLaunch L{};
      L.kind = pass == 0 ? 1 : 2;
      L.pl = pl;
      L.probs = ring.put(gp.data(), sizeof(Params) * gp.size(), s);
      L.off = static_cast<const int64_t*>(ring.put(off.data(), sizeof(int64_t) * off.size(), s));
      L.n = static_cast<int>(gp.size());
      L.total = total;
      L.blocks = static_cast<int>(std::min<int64_t>(4LL * sm_count_current(), std::max<int64_t>(1, (total + 255) / 256)));
      plan.launches.push_back(L);
    }
}

void grouped_exec(const GroupedPlan& plan, cudaStream_t s, int64_t* launches) {
  int ngemm = 0;
  for (const GroupedLaunch& L : plan.launches) ngemm += L.kind == 0 ? 1 : 0;
  SideStreams* ss = ngemm > 1 ? plan.side : nullptr;
  if (ss) ss->make();
  if (ss) RR_CUDA(cudaEventRecord(ss->fork, s));
  int k = 0;
  bool joined = ss == nullptr;
  for (const GroupedLaunch& L : plan.launches) {
    GroupArgs g;
    g.probs = static_cast<const Params*>(L.probs);
    g.off = L.off;
    g.n = L.n;
    g.total = L.total;
    if (L.kind == 0) {
      cudaStream_t t = s;
      if (ss) {
        t = ss->st[k % SideStreams::kCount];
        if (k < SideStreams::kCount) RR_CUDA(cudaStreamWaitEvent(t, ss->fork, 0));
        ++k;
      }
      launch_cfg(L.cplx, L.AK, L.BKM, L.cfg, L.vec2, g, t);
    } else {
      if (!joined) {  // the tile launches (all before the first reduction in a plan) are done first
        for (int i = 0; i < std::min(k, SideStreams::kCount); ++i) {
          RR_CUDA(cudaEventRecord(ss->done[i], ss->st[i]));
          RR_CUDA(cudaStreamWaitEvent(s, ss->done[i], 0));
        }
        joined = true;
      }
      if (L.kind == 1) {
        if (L.pl == 2) splitk_reduce_grouped_kernel<2><<<L.blocks, 256, 0, s>>>(g);
        else splitk_reduce_grouped_kernel<1><<<L.blocks, 256, 0, s>>>(g);
      } else {
        if (L.pl == 2) mirror_grouped_kernel<2><<<L.blocks, 256, 0, s>>>(g);
        else mirror_grouped_kernel<1><<<L.blocks, 256, 0, s>>>(g);
      }
      RR_LAUNCH_CHECK();
    }
    if (launches) ++*launches;
  }
  if (!joined)
    for (int i = 0; i < std::min(k, SideStreams::kCount); ++i) {
      RR_CUDA(cudaEventRecord(ss->done[i], ss->st[i]));
      RR_CUDA(cudaStreamWaitEvent(s, ss->done[i], 0));
    }
}

void grouped_run(const std::vector<GemmDesc>& descs, const std::vector<GemmChoice>& choice, cudaStream_t s,
                 TableRing& ring, DevBuf<double>& work, int64_t* launches) {
  GroupedPlan plan;
  grouped_build(descs, choice, s, ring, work, plan);
  grouped_exec(plan, s, launches);
}

// ------------------------------------------------------------------------------------ autotuner

int64_t bucket(int64_t x) {
  if (x <= 64) return round_up(std::max<int64_t>(x, 1), 8);
  if (x <= 512) return round_up(x, 32);
  if (x <= 4096) return round_up(x, 256);
  return round_up(x, 2048);
}

// Cache key: element kind, layout, mirror mode and the bucketed M, N, K, batch.
struct ShapeKey {
  int64_t v[8];
  bool operator==(const ShapeKey& o) const {
    for (int i = 0; i < 8; ++i)
      if (v[i] != o.v[i]) return false;
    return true;
  }
};

struct ShapeKeyHash {
  size_t operator()(const ShapeKey& k) const {
    uint64_t h = 1469598103934665603ull;
    for (int i = 0; i < 8; ++i) h = (h ^ static_cast<uint64_t>(k.v[i])) * 1099511628211ull;
    return static_cast<size_t>(h);
  }
};

ShapeKey shape_key(const GemmDesc& d) {
  return ShapeKey{{d.cplx ? 1 : 0, static_cast<int64_t>(d.opA), static_cast<int64_t>(d.opB), d.mirror, bucket(d.M),
                   bucket(d.N), bucket(d.K), bucket(d.batch)}};
}

// The cache file's text form of a key: c<kind>a<opA>b<opB>m<mirror>_<M>x<N>x<K>x<batch>.
std::string key_text(const ShapeKey& k) {
  std::ostringstream t;
  t << "c" << k.v[0] << "a" << k.v[1] << "b" << k.v[2] << "m" << k.v[3] << "_" << k.v[4] << "x" << k.v[5] << "x" << k.v[6]
    << "x" << k.v[7];
  return t.str();
}

bool parse_key(const std::string& s, ShapeKey& k) {
  long long v[8];
  if (std::sscanf(s.c_str(), "c%llda%lldb%lldm%lld_%lldx%lldx%lldx%lld", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6],
                  &v[7]) != 8)
    return false;
  for (int i = 0; i < 8; ++i) k.v[i] = v[i];
  return true;
}

// Doubles spanned by the output of d (every batch entry, plane and mirrored triangle).
int64_t c_extent(const GemmDesc& d) {
  const int64_t rows = d.c_plane_rows > 0 ? std::min(d.M, d.c_plane_rows) : d.M;
  const int64_t planes = d.c_plane_rows > 0 ? ((d.M - 1) / d.c_plane_rows) * d.c_plane_stride : 0;
  int64_t last = planes + (d.batch - 1) * d.strideC + (rows - 1) * d.ldc + (d.N - 1) * d.c_col_stride;
  if (d.mirror) last = std::max(last, (d.batch - 1) * d.strideC + (d.N - 1) * d.ldc + (d.M - 1));
  return (d.cplx ? 2 : 1) * (last + 1);
}

std::vector<int> candidate_cfgs(const GemmDesc& d) {
  if (d.cplx) return {0, 1};
  if (d.M <= 8) return {3, 4, 0};
  if (d.M <= 16) return {4, 0};
  if (d.M <= 32) return {5, 0, 6};
  if (d.M <= 40) return {6, 0, 1};
  return {0, 1, 2};
}

struct Tuner {
  std::mutex mu;
  std::unordered_map<ShapeKey, std::pair<GemmChoice, double>, ShapeKeyHash> cache;
  bool env_loaded = false, dirty = false;
  TableRing ring;
  DevBuf<double> cbuf, wbuf;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  double seconds = 0.0;
  int64_t launches = 0;
};

Tuner& tuner() {
  static Tuner* t = new Tuner();  // never destroyed: no CUDA calls during static destruction
  return *t;
}

void load_locked(Tuner& t, const std::string& path) {
  std::ifstream in(path);
  if (!in) return;
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ls(line);
    std::string text;
    GemmChoice c;
    double us = 0.0;
    ShapeKey key;
    if (!(ls >> text >> c.cfg >> c.splits >> us) || !parse_key(text, key)) continue;
    if (c.cfg < 0 || c.cfg > 6 || c.splits < 1 || c.splits > 64) continue;
    if (key.v[0] == 1 && c.cfg > 1) continue;  // complex products have two configurations
    t.cache[key] = {c, us};
  }
}

void save_locked(Tuner& t, const std::string& path) {
  std::map<std::string, std::pair<GemmChoice, double>> sorted;
  for (auto& [k, v] : t.cache) sorted[key_text(k)] = v;
  const std::string tmp = path + ".tmp";
  {
    std::ofstream out(tmp, std::ios::trunc);
    if (!out) throw Error(RR_ERR_ARG, "autotune: cannot write " + tmp);
    for (auto& [k, v] : sorted) out << k << " " << v.first.cfg << " " << v.first.splits << " " << v.second << "\n";
  }
  if (std::rename(tmp.c_str(), path.c_str()) != 0) throw Error(RR_ERR_ARG, "autotune: cannot replace " + path);
  t.dirty = false;
}

void env_load_locked(Tuner& t) {
  if (t.env_loaded) return;
  t.env_loaded = true;
  if (const char* p = std::getenv("RR_AUTOTUNE_CACHE")) load_locked(t, p);
}

// Device time per problem of `cand` for d: a grouped launch of R copies of d (shared inputs, separate
// outputs and split-K scratch), R chosen so that the copies fill the GPU about twice.
double measure(Tuner& t, const GemmDesc& d, GemmChoice cand) {
  const TileDims td = dims_of(d.cplx, cand.cfg);
  int64_t tiles = static_cast<int64_t>(ceil_div(d.M, td.bm)) * ceil_div(d.N, td.bn) * d.batch * cand.splits;
  if (d.mirror) tiles = (tiles + ceil_div(d.M, td.bm) * d.batch * cand.splits) / 2;
  const int64_t want = 8LL * sm_count_current();
  int64_t R = std::max<int64_t>(1, std::min<int64_t>(64, (want + tiles - 1) / std::max<int64_t>(tiles, 1)));
  const int64_t cext = round_up(c_extent(d), 32);
  const int64_t wsz = cand.splits > 1 ? d.batch * cand.splits * d.M * d.N * (d.cplx ? 2 : 1) : 0;
  while (R > 1 && R * (cext + wsz) > (int64_t{32} << 20)) R /= 2;
  if (static_cast<int64_t>(t.cbuf.n) < R * cext) {
    t.cbuf.alloc(static_cast<size_t>(R * cext));
    RR_CUDA(cudaMemsetAsync(t.cbuf.p, 0, sizeof(double) * R * cext, t.s));
  }
  std::vector<GemmDesc> copies(static_cast<size_t>(R), d);
  for (int64_t r = 0; r < R; ++r) copies[r].C = t.cbuf.p + r * cext;
  std::vector<GemmChoice> ch(static_cast<size_t>(R), cand);
  grouped_run(copies, ch, t.s, t.ring, t.wbuf, nullptr);  // warm-up (and scratch growth)
  RR_CUDA(cudaStreamSynchronize(t.s));
  t.ring.reset();
  constexpr int reps = 3;
  RR_CUDA(cudaEventRecord(t.e0, t.s));
  for (int k = 0; k < reps; ++k) grouped_run(copies, ch, t.s, t.ring, t.wbuf, nullptr);
  RR_CUDA(cudaEventRecord(t.e1, t.s));
  RR_CUDA(cudaEventSynchronize(t.e1));
  t.ring.reset();
  float ms = 0.f;
  RR_CUDA(cudaEventElapsedTime(&ms, t.e0, t.e1));
  return 1e3 * ms / (reps * static_cast<double>(R));
}

}  // namespace

SideStreams::~SideStreams() {
  for (int i = 0; i < kCount; ++i) {
    if (st[i]) cudaStreamDestroy(st[i]);
    if (done[i]) cudaEventDestroy(done[i]);
  }
  if (fork) cudaEventDestroy(fork);
}

void SideStreams::make() {
  if (fork) return;
  for (int i = 0; i < kCount; ++i) {
    RR_CUDA(cudaStreamCreateWithFlags(&st[i], cudaStreamNonBlocking));
    RR_CUDA(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
  }
  RR_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
}

TableRing::~TableRing() {
  if (host) cudaFreeHost(host);
  for (auto& r : retired) cudaFreeHost(r.second);
}

void TableRing::reserve(size_t bytes) {
  if (bytes <= cap) return;
  if (host) retired.emplace_back(std::move(dev), host);
  host = nullptr;
  RR_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host), bytes));
  dev.alloc(bytes);
  cap = bytes;
  used = 0;
}

void TableRing::reset() {
  used = 0;
  for (auto& r : retired) {
    cudaFreeHost(r.second);
    r.first.release();
  }
  retired.clear();
}

const void* TableRing::put(const void* src, size_t bytes, cudaStream_t s) {
  RR_REQUIRE(src && bytes > 0, RR_ERR_ARG, "TableRing::put: empty table");
  const size_t need = (bytes + 15) & ~size_t{15};
  if (cap == 0) reserve(std::max<size_t>(size_t{4} << 20, 2 * need));
  else if (used + need > cap) reserve(std::max(2 * cap, 2 * need));
  std::memcpy(host + used, src, bytes);
  RR_CUDA(cudaMemcpyAsync(dev.p + used, host + used, bytes, cudaMemcpyHostToDevice, s));
  const void* out = dev.p + used;
  used += need;
  return out;
}

void gemm_grouped_plan(const std::vector<GemmDesc>& descs, cudaStream_t s, TableRing& ring, DevBuf<double>& work,
                       GroupedPlan& plan) {
  std::vector<GemmChoice> ch;
  autotune_choices(descs, ch);
  grouped_build(descs, ch, s, ring, work, plan);
}

void gemm_grouped_exec(const GroupedPlan& plan, cudaStream_t s, int64_t* launches) { grouped_exec(plan, s, launches); }

void gemm_grouped(const std::vector<GemmDesc>& descs, cudaStream_t s, TableRing& ring, DevBuf<double>& work,
                  int64_t* launches) {
  std::vector<GemmChoice> ch;
  autotune_choices(descs, ch);
  grouped_run(descs, ch, s, ring, work, launches);
}

namespace {
GemmChoice choice_locked(Tuner& t, const GemmDesc& d);
}  // namespace

GemmChoice autotune_choice(const GemmDesc& d) {
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  return choice_locked(t, d);
}

void autotune_choices(const std::vector<GemmDesc>& descs, std::vector<GemmChoice>& out) {
  out.assign(descs.size(), GemmChoice{});
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  for (size_t i = 0; i < descs.size(); ++i)
    if (descs[i].M > 0 && descs[i].N > 0 && descs[i].batch > 0) out[i] = choice_locked(t, descs[i]);
}

namespace {
GemmChoice choice_locked(Tuner& t, const GemmDesc& d) {
  env_load_locked(t);
  const ShapeKey key = shape_key(d);
  auto it = t.cache.find(key);
  if (it != t.cache.end()) return it->second.first;
  if (!t.s) {
    RR_CUDA(cudaStreamCreateWithFlags(&t.s, cudaStreamNonBlocking));
    RR_CUDA(cudaEventCreate(&t.e0));
    RR_CUDA(cudaEventCreate(&t.e1));
  }
  const auto t0 = std::chrono::steady_clock::now();
  const int64_t l0 = rr::launches();
  GemmChoice best;
  double best_us = 1e300;
  for (int cfg : candidate_cfgs(d)) {
    for (int sp : {1, 2, 4, 8, 16}) {
      if (sp > 1 && d.K < static_cast<int64_t>(sp) * 4 * gk::KT) break;
      const GemmChoice c{cfg, sp};
      const double us = measure(t, d, c);
      if (us < best_us) {
        best_us = us;
        best = c;
      }
    }
  }
  t.cache[key] = {best, best_us};
  t.dirty = true;
  t.seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  t.launches += rr::launches() - l0;
  return best;
}
}  // namespace

void autotune_load(const std::string& path) {
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  t.env_loaded = true;
  load_locked(t, path);
}

void autotune_save(const std::string& path) {
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  save_locked(t, path);
}

void autotune_flush() {
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  const char* p = std::getenv("RR_AUTOTUNE_CACHE");
  if (p && t.dirty) save_locked(t, p);
}

void autotune_clear() {
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  t.cache.clear();
  t.dirty = false;
}

void autotune_totals(double* seconds, int64_t* launches) {
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  if (seconds) *seconds = t.seconds;
  if (launches) *launches = t.launches;
}

int64_t autotune_entries() {
  Tuner& t = tuner();
  std::lock_guard<std::mutex> lk(t.mu);
  return static_cast<int64_t>(t.cache.size());
}

}  // namespace rr
