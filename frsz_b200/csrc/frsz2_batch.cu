// frsz2_batch.cu -- many arrays of mixed float types, widths and sizes per
// call: one CUDA graph launch whose parallel branches are one kernel per
// (float type, width) class present in the batch, over the class's
// device-resident work list: one CTA per tile (the tile's array from a
// per-tile index; the default) or a persistent grid walking the class's
// tiles.  An autotuner picks between them, and the CTA shape, the number of
// resident CTAs per SM of the persistent grid and whether classes run side by
// side or one after another, by timing the candidates on the plan's own
// arrays.
//
// One kernel per class rather than one kernel switching over widths: a
// multi-width kernel gets a register allocation sized for the union of its
// cases (237-255 registers for 13-18 widths measured with ptxas -v, against
// 40-64 for any single width), which would cut occupancy to a quarter.
#include "frsz2_batch_kernels.cuh"
#include "frsz2_launch.hpp"

#include "../../include/frsz2_b200.h"

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

using namespace frsz2b;

namespace {

struct Class
{
  int is64 = 0, bits = 0;
  std::vector<int> items;                         // plan item indices
  std::uint64_t tiles[kNumShapes] = { 0, 0, 0 };
  std::size_t desc_off[kNumShapes] = { 0, 0, 0 }; // first descriptor in the shape's array
  std::uint64_t tmap_off = 0;                     // first entry of the shape-0 tile index
  batch_entry entry[kNumShapes] = {};
};

constexpr int kMaxBranches = 16;

} // namespace

// Opaque plan behind the C ABI.
struct frsz2_batch
{
  std::vector<frsz2_batch_item> items;
  std::vector<Class> classes;
  std::vector<int> other_items; // items with their own launch
  BatchItem* d_desc[kNumShapes] = { nullptr, nullptr, nullptr };
  // shape 0, per tile of every class: the tile's descriptor within its class
  std::uint32_t* d_tmap = nullptr;
  bool shape_ok[kNumShapes] = { false, false, false };
  // launch configuration per direction (0 = decompress, 1 = compress)
  int shape[2] = { 0, 0 };
  int ctas_per_sm[2] = { 0, 0 };
  int parallel[2] = { 1, 1 };
  int per_tile[2] = { 0, 0 }; // 1: one CTA per tile (shape 0), not the persistent class kernels
  bool tuned[2] = { false, false };
  cudaGraphExec_t graph[2] = { nullptr, nullptr };
  cudaStream_t branch[kMaxBranches] = {};
  cudaEvent_t fork = nullptr, join[kMaxBranches] = {};
  std::mutex mu;
};

namespace {

std::uint64_t class_tiles_total(const frsz2_batch* p, int shape)
{
  std::uint64_t t = 0;
  for (const auto& c : p->classes) t += c.tiles[shape];
  return t;
}

int min_occupancy(const frsz2_batch* p, int shape, bool compress)
{
  int occ = 64;
  for (const auto& c : p->classes) occ = std::min(occ, c.entry[shape].occupancy(compress));
  return std::max(1, occ);
}

int ensure_branches(frsz2_batch* p)
{
  if (p->fork) return FRSZ2_OK;
  if (int rc = cuda_status(cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming), "event create")) return rc;
  for (int i = 0; i < kMaxBranches; ++i) {
    if (int rc = cuda_status(cudaStreamCreateWithFlags(&p->branch[i], cudaStreamNonBlocking), "stream create"))
      return rc;
    if (int rc = cuda_status(cudaEventCreateWithFlags(&p->join[i], cudaEventDisableTiming), "event create"))
      return rc;
  }
  return FRSZ2_OK;
}

// Enqueue one direction on stream s with the given configuration; per_tile
// launches one CTA per tile of each class (shape 0) instead of the
// persistent class kernels.
int enqueue(frsz2_batch* p, bool compress, cudaStream_t s, int shape, int ctas_per_sm, bool parallel,
            bool per_tile = false)
{
  const std::uint64_t total = class_tiles_total(p, shape);
  const std::uint64_t ctas = (std::uint64_t)sm_count() * (std::uint64_t)ctas_per_sm;
  const int nb = std::min<int>((int)p->classes.size(), kMaxBranches);
  const bool fork = parallel && nb > 1;
  if (fork) {
    if (int rc = cuda_status(cudaEventRecord(p->fork, s), "fork")) return rc;
    for (int b = 0; b < nb; ++b)
      if (int rc = cuda_status(cudaStreamWaitEvent(p->branch[b], p->fork, 0), "fork wait")) return rc;
  }
  for (std::size_t ci = 0; ci < p->classes.size(); ++ci) {
    const Class& c = p->classes[ci];
    const std::uint64_t tiles = c.tiles[shape];
    if (tiles == 0) continue;
    // side by side: each class gets its share of the resident CTAs
    std::uint64_t grid = fork ? (ctas * tiles + total - 1) / total : ctas;
    grid = std::max<std::uint64_t>(1, std::min(grid, tiles));
    cudaStream_t st = fork ? p->branch[ci % nb] : s;
    const cudaError_t e =
      per_tile && shape == 0 && c.entry[0].launch_tiles && p->d_tmap
        ? c.entry[0].launch_tiles(compress, p->d_desc[0] + c.desc_off[0], p->d_tmap + c.tmap_off, tiles, st)
        : c.entry[shape].launch(compress, p->d_desc[shape] + c.desc_off[shape], (int)c.items.size(), tiles,
                                (unsigned)grid, st);
    if (int rc = cuda_status(e, "batch launch")) return rc;
  }
  if (fork) {
    for (int b = 0; b < nb; ++b) {
      if (int rc = cuda_status(cudaEventRecord(p->join[b], p->branch[b]), "join")) return rc;
      if (int rc = cuda_status(cudaStreamWaitEvent(s, p->join[b], 0), "join wait")) return rc;
    }
  }
  for (int i : p->other_items) {
    const frsz2_batch_item& it = p->items[i];
    const Layout L = make_layout(it.n, it.bits, it.block_size);
    Job j = job_for_slice(L, it.dtype, 0, L.nb, it.values, it.decompressed, static_cast<std::uint8_t*>(it.compressed));
    const int rc = compress ? launch_compress(j, it.dtype, s, nullptr) : launch_decompress(j, it.dtype, s, nullptr);
    if (rc) return rc;
  }
  return FRSZ2_OK;
}

int build_graph(frsz2_batch* p, bool compress)
{
  const int d = compress ? 1 : 0;
  if (p->graph[d]) {
    cudaGraphExecDestroy(p->graph[d]);
    p->graph[d] = nullptr;
  }
  cudaStream_t cs = nullptr;
  int rc = cuda_status(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking), "stream create");
  if (rc) return rc;
  cudaGraph_t g = nullptr;
  rc = cuda_status(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal), "begin capture");
  if (!rc) {
    rc = enqueue(p, compress, cs, p->shape[d], p->ctas_per_sm[d], p->parallel[d] != 0, p->per_tile[d] != 0);
    const int rc2 = cuda_status(cudaStreamEndCapture(cs, &g), "end capture");
    if (!rc) rc = rc2;
  }
  if (!rc) rc = cuda_status(cudaGraphInstantiate(&p->graph[d], g, 0), "graph instantiate");
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  return rc;
}

// Untuned configuration: what the autotuner picked for the 4096-array mixed
// batch: one CTA per tile (256 x 2), classes side by side (0.95 of HBM, against
// 0.90 for the persistent class kernels, 4 resident CTAs per SM, classes one
// after another, which the autotuner picked before the per-tile launch
// existed).  Plans without the tile index keep the persistent kernels.
void default_config(frsz2_batch* p, bool compress)
{
  const int d = compress ? 1 : 0;
  p->shape[d] = 0;
  p->ctas_per_sm[d] = p->classes.empty() ? 1 : std::min(4, min_occupancy(p, 0, compress));
  p->per_tile[d] = p->d_tmap && p->shape_ok[0] ? 1 : 0;
  p->parallel[d] = p->per_tile[d];
}

int check_direction(const frsz2_batch* p, bool compress)
{
  for (const auto& it : p->items)
    if (it.n > 0 && (compress ? it.values == nullptr : it.decompressed == nullptr))
      return set_error(FRSZ2_EFAIL, compress ? "batch item without values: plan is decompress-only"
                                             : "batch item without an output array: plan is compress-only");
  return FRSZ2_OK;
}

int run(frsz2_batch* p, bool compress, cudaStream_t s)
{
  std::lock_guard<std::mutex> lock(p->mu);
  if (int rc = check_direction(p, compress)) return rc;
  const int d = compress ? 1 : 0;
  if (p->ctas_per_sm[d] == 0) default_config(p, compress);
  if (!p->graph[d])
    if (int rc = build_graph(p, compress)) return rc;
  return cuda_status(cudaGraphLaunch(p->graph[d], s), "graph launch");
}

// Time every (shape, CTAs per SM, side by side or one after another) on the
// plan's arrays; keep the fastest and rebuild that direction's graph.
int autotune(frsz2_batch* p, bool compress, cudaStream_t s, float* best_ms_out)
{
  const int d = compress ? 1 : 0;
  cudaEvent_t a, b;
  int rc = cuda_status(cudaEventCreate(&a), "event create");
  if (rc) return rc;
  if ((rc = cuda_status(cudaEventCreate(&b), "event create"))) {
    cudaEventDestroy(a);
    return rc;
  }
  float best = 1e30f;
  int best_shape = p->shape[d], best_ctas = p->ctas_per_sm[d], best_par = p->parallel[d], best_tile = p->per_tile[d];
  const int modes = p->classes.size() > 1 ? 2 : 1;
  for (int shape = 0; shape < kNumShapes && !rc; ++shape) {
    if (!p->shape_ok[shape] || p->classes.empty()) continue;
    const int occ = min_occupancy(p, shape, compress);
    for (int m = 0; m < modes && !rc; ++m) {
      const bool par = m == 0;
      for (int c : { 1, 2, 3, 4, 6, 8, 12, 16 }) {
        if (c > occ) break;
        if ((rc = enqueue(p, compress, s, shape, c, par))) break; // warm
        float ms_min = 1e30f;
        for (int rep = 0; rep < 3 && !rc; ++rep) {
          cudaEventRecord(a, s);
          rc = enqueue(p, compress, s, shape, c, par);
          cudaEventRecord(b, s);
          if (!rc) rc = cuda_status(cudaEventSynchronize(b), "autotune sync");
          float ms = 0;
          if (!rc) cudaEventElapsedTime(&ms, a, b);
          ms_min = std::min(ms_min, ms);
        }
        if (rc) break;
        if (ms_min < best) {
          best = ms_min;
          best_shape = shape;
          best_ctas = c;
          best_par = par ? 1 : 0;
          best_tile = 0;
        }
      }
    }
  }
  // one CTA per tile (shape 0), classes side by side or one after another
  for (int m = 0; m < modes && !rc && p->d_tmap && p->shape_ok[0] && !p->classes.empty(); ++m) {
    const bool par = m == 0;
    if ((rc = enqueue(p, compress, s, 0, 1, par, true))) break; // warm
    float ms_min = 1e30f;
    for (int rep = 0; rep < 3 && !rc; ++rep) {
      cudaEventRecord(a, s);
      rc = enqueue(p, compress, s, 0, 1, par, true);
      cudaEventRecord(b, s);
      if (!rc) rc = cuda_status(cudaEventSynchronize(b), "autotune sync");
      float ms = 0;
      if (!rc) cudaEventElapsedTime(&ms, a, b);
      ms_min = std::min(ms_min, ms);
    }
    if (!rc && ms_min < best) {
      best = ms_min;
      best_shape = 0;
      best_ctas = p->ctas_per_sm[d];
      best_par = par ? 1 : 0;
      best_tile = 1;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (rc) return rc;
  p->shape[d] = best_shape;
  p->ctas_per_sm[d] = best_ctas;
  p->parallel[d] = best_par;
  p->per_tile[d] = best_tile;
  p->tuned[d] = true;
  if (best_ms_out) *best_ms_out = best;
  return build_graph(p, compress);
}

} // namespace

extern "C" {

int frsz2_batch_create(const frsz2_batch_item* items, uint64_t count, frsz2_batch** plan)
{
  if (!plan) return set_error(FRSZ2_EFAIL, "null plan pointer");
  *plan = nullptr;
  if (count > 0 && !items) return set_error(FRSZ2_EFAIL, "null items");
  auto* p = new frsz2_batch();
  p->items.assign(items, items + count);
  for (std::uint64_t i = 0; i < count; ++i) {
    const frsz2_batch_item& it = p->items[i];
    int rc = check_args(it.dtype, it.bits, it.block_size);
    if (!rc && it.n > 0 && (!it.compressed || (!it.values && !it.decompressed)))
      rc = set_error(FRSZ2_EFAIL, "null pointer in batch item " + std::to_string(i));
    const std::uintptr_t es = it.dtype == FRSZ2_DOUBLE ? 8 : 4;
    const std::uintptr_t ws = (std::uintptr_t)word_bits(it.bits) / 8;
    if (!rc && it.n > 0 &&
        (reinterpret_cast<std::uintptr_t>(it.values) % es != 0 ||
         reinterpret_cast<std::uintptr_t>(it.decompressed) % es != 0 ||
         reinterpret_cast<std::uintptr_t>(it.compressed) % ws != 0))
      rc = set_error(FRSZ2_EFAIL, "misaligned pointer in batch item " + std::to_string(i));
    if (rc) {
      delete p;
      return rc;
    }
    if (it.n == 0) continue;
    const bool is64 = it.dtype == FRSZ2_DOUBLE;
    const Layout L = make_layout(it.n, it.bits, it.block_size);
    Job j = job_for_slice(L, it.dtype, 0, L.nb, it.values, it.decompressed, static_cast<std::uint8_t*>(it.compressed));
    const batch_entry e0 = is64 ? batch_class_f64(it.bits, 0) : batch_class_f32(it.bits, 0);
    const bool ok = e0.launch && (!it.values || fast_eligible(j, is64, it.values, j.words)) &&
                    (!it.decompressed || fast_eligible(j, is64, it.decompressed, j.words));
    if (!ok) {
      p->other_items.push_back((int)i);
      continue;
    }
    auto c = std::find_if(p->classes.begin(), p->classes.end(),
                          [&](const Class& k) { return k.is64 == (int)is64 && k.bits == it.bits; });
    if (c == p->classes.end()) {
      Class k;
      k.is64 = is64;
      k.bits = it.bits;
      for (int sh = 0; sh < kNumShapes; ++sh)
        k.entry[sh] = is64 ? batch_class_f64(it.bits, sh) : batch_class_f32(it.bits, sh);
      p->classes.push_back(k);
      c = p->classes.end() - 1;
    }
    c->items.push_back((int)i);
  }
  for (int sh = 0; sh < kNumShapes; ++sh) {
    std::vector<BatchItem> desc;
    bool ok = !p->classes.empty();
    for (auto& c : p->classes) {
      if (!c.entry[sh].launch) ok = false;
      c.desc_off[sh] = desc.size();
      std::uint64_t tb = 0;
      for (int i : c.items) {
        const frsz2_batch_item& it = p->items[i];
        const int tv = fast_tile_values(c.is64 ? 8 : 4, kShapes[sh].nt, kShapes[sh].rpw);
        if (it.block_size > tv) ok = false;
        const Layout L = make_layout(it.n, it.bits, it.block_size);
        BatchItem bi{};
        bi.job = job_for_slice(L, it.dtype, 0, L.nb, it.values, it.decompressed,
                               static_cast<std::uint8_t*>(it.compressed));
        bi.job.tiles = (it.n + (std::uint64_t)tv - 1) / (std::uint64_t)tv;
        bi.job.tile_blocks = (std::uint32_t)(tv / it.block_size);
        bi.tile_begin = tb;
        tb += bi.job.tiles;
        desc.push_back(bi);
      }
      c.tiles[sh] = tb;
    }
    p->shape_ok[sh] = ok;
    if (!ok) continue;
    int rc = cuda_status(cudaMalloc(&p->d_desc[sh], desc.size() * sizeof(BatchItem)), "descriptor allocation");
    if (!rc)
      rc = cuda_status(cudaMemcpy(p->d_desc[sh], desc.data(), desc.size() * sizeof(BatchItem), cudaMemcpyHostToDevice),
                       "descriptor upload");
    if (rc) {
      frsz2_batch_destroy(p);
      return rc;
    }
  }
  if (p->shape_ok[0]) {
    std::vector<std::uint32_t> tmap;
    for (auto& c : p->classes) {
      c.tmap_off = tmap.size();
      for (std::size_t k = 0; k < c.items.size(); ++k) {
        const frsz2_batch_item& it = p->items[c.items[k]];
        const int tv = fast_tile_values(c.is64 ? 8 : 4, kShapes[0].nt, kShapes[0].rpw);
        tmap.insert(tmap.end(), (it.n + (std::uint64_t)tv - 1) / (std::uint64_t)tv, (std::uint32_t)k);
      }
    }
    int rc = cuda_status(cudaMalloc(&p->d_tmap, std::max<std::size_t>(1, tmap.size()) * sizeof(std::uint32_t)),
                         "tile index allocation");
    if (!rc && !tmap.empty())
      rc = cuda_status(cudaMemcpy(p->d_tmap, tmap.data(), tmap.size() * sizeof(std::uint32_t), cudaMemcpyHostToDevice),
                       "tile index upload");
    if (rc) {
      frsz2_batch_destroy(p);
      return rc;
    }
  }
  if (!p->classes.empty() && !p->shape_ok[0]) {
    // block sizes too large for the default tile: every array gets its own launch
    for (auto& c : p->classes) p->other_items.insert(p->other_items.end(), c.items.begin(), c.items.end());
    p->classes.clear();
  }
  if (int rc = ensure_branches(p)) {
    frsz2_batch_destroy(p);
    return rc;
  }
  *plan = p;
  return FRSZ2_OK;
}

int frsz2_batch_compress(frsz2_batch* plan, void* stream)
{
  NvtxRange nvtx("frsz2_batch_compress");
  if (!plan) return set_error(FRSZ2_EFAIL, "null plan");
  return run(plan, true, static_cast<cudaStream_t>(stream));
}

int frsz2_batch_decompress(frsz2_batch* plan, void* stream)
{
  NvtxRange nvtx("frsz2_batch_decompress");
  if (!plan) return set_error(FRSZ2_EFAIL, "null plan");
  return run(plan, false, static_cast<cudaStream_t>(stream));
}

int frsz2_batch_autotune(frsz2_batch* plan, int compress, void* stream, float* best_ms)
{
  NvtxRange nvtx("frsz2_batch_autotune");
  if (!plan) return set_error(FRSZ2_EFAIL, "null plan");
  std::lock_guard<std::mutex> lock(plan->mu);
  if (int rc = check_direction(plan, compress != 0)) return rc;
  if (plan->ctas_per_sm[compress ? 1 : 0] == 0) default_config(plan, compress != 0);
  return autotune(plan, compress != 0, static_cast<cudaStream_t>(stream), best_ms);
}

int frsz2_batch_configure(frsz2_batch* plan, int compress, int shape, int ctas_per_sm, int side_by_side,
                          int one_cta_per_tile)
{
  if (!plan) return set_error(FRSZ2_EFAIL, "null plan");
  std::lock_guard<std::mutex> lock(plan->mu);
  if (shape < 0 || shape >= kNumShapes || !plan->shape_ok[shape])
    return set_error(FRSZ2_EFAIL, "launch shape " + std::to_string(shape) + " is not available for this plan");
  if (one_cta_per_tile && (shape != 0 || !plan->d_tmap))
    return set_error(FRSZ2_EFAIL, "one CTA per tile needs launch shape 0");
  const int occ = plan->classes.empty() ? 1 : min_occupancy(plan, shape, compress != 0);
  if (ctas_per_sm < 1 || ctas_per_sm > occ)
    return set_error(FRSZ2_EFAIL, "ctas_per_sm must be 1.." + std::to_string(occ) + " for this plan and shape");
  const int d = compress ? 1 : 0;
  plan->shape[d] = shape;
  plan->ctas_per_sm[d] = ctas_per_sm;
  plan->parallel[d] = side_by_side ? 1 : 0;
  plan->per_tile[d] = one_cta_per_tile ? 1 : 0;
  plan->tuned[d] = false;
  return build_graph(plan, compress != 0);
}

int frsz2_batch_info(const frsz2_batch* plan, frsz2_batch_stats* out)
{
  if (!plan || !out) return set_error(FRSZ2_EFAIL, "null pointer");
  std::memset(out, 0, sizeof(*out));
  out->arrays = plan->items.size();
  for (const auto& c : plan->classes) out->persistent_arrays += c.items.size();
  out->separate_launches = plan->other_items.size();
  out->classes = plan->classes.size();
  for (int d = 0; d < 2; ++d) {
    const int sh = plan->shape[d];
    out->threads_per_cta[d] = kShapes[sh].nt;
    out->rows_per_warp[d] = kShapes[sh].rpw;
    out->ctas_per_sm[d] = plan->ctas_per_sm[d];
    out->side_by_side[d] = plan->parallel[d];
    out->tiles[d] = class_tiles_total(plan, sh);
    out->tuned[d] = plan->tuned[d] ? 1 : 0;
    out->one_cta_per_tile[d] = plan->per_tile[d];
  }
  return FRSZ2_OK;
}

void frsz2_batch_destroy(frsz2_batch* plan)
{
  if (!plan) return;
  for (auto& g : plan->graph)
    if (g) cudaGraphExecDestroy(g);
  for (auto& d : plan->d_desc)
    if (d) cudaFree(d);
  if (plan->d_tmap) cudaFree(plan->d_tmap);
  for (int i = 0; i < kMaxBranches; ++i) {
    if (plan->branch[i]) cudaStreamDestroy(plan->branch[i]);
    if (plan->join[i]) cudaEventDestroy(plan->join[i]);
  }
  if (plan->fork) cudaEventDestroy(plan->fork);
  delete plan;
}

} // extern "C"
