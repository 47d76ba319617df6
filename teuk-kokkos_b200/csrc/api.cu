// C ABI of the B200 engine (include/teuk_b200.h).  A pipeline is a batch of
// one solve; a batch packs many independent solves of uneven shape into the
// same four stage launches per RK4 step.  Host code here validates, plans,
// owns device memory and orders launches on one CUDA stream; it never
// computes a right-hand side itself.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <deque>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <numbers>
#include <stdexcept>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "kernels.h"
#include "checkpoint.h"
#include "run_config.h"
#include "second_order.h"
#include "split_precision.cuh"
#include "static_scratch.h"
#include "teuk_b200.h"

namespace teuk_b200 {
namespace {

thread_local std::string g_last_error;

// Failure-detection test hook (teuk_b200_test_withhold_chunk): the chunk
// that CTA 0's producer skips in stage-1 launches of batches built while it
// is set; -1 (the default) disables it.
std::atomic<int> g_test_withhold_chunk{-1};

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct Unsupported : std::runtime_error {
  using std::runtime_error::runtime_error;
};

void check(const cudaError_t err, const char* what) {
  if (err != cudaSuccess) {
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(err));
  }
}

template <class Body>
int guarded(Body&& body) {
  try {
    body();
    return TEUK_B200_OK;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return TEUK_B200_ERR_INVALID_ARGUMENT;
  } catch (const std::out_of_range& e) {
    g_last_error = e.what();
    return TEUK_B200_ERR_INVALID_ARGUMENT;
  } catch (const Unsupported& e) {
    g_last_error = e.what();
    return TEUK_B200_ERR_UNSUPPORTED;
  } catch (const CudaError& e) {
    g_last_error = e.what();
    return TEUK_B200_ERR_CUDA;
  } catch (const DeviceError& e) {
    g_last_error = e.what();
    return TEUK_B200_ERR_CUDA;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return TEUK_B200_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return TEUK_B200_ERR_RUNTIME;
  }
}

Config to_config(const teuk_b200_config& c) {
  if (c.abi_version != TEUK_B200_ABI_VERSION) {
    throw std::invalid_argument("teuk_b200_config.abi_version mismatch");
  }
  const auto list = [](const int* values, const int count) {
    if (count < 0 || (count > 0 && values == nullptr)) {
      throw std::invalid_argument("mode list pointer/count mismatch");
    }
    return std::vector<int>(values, values + count);
  };
  Config out;
  out.mass = c.mass;
  out.spin = c.spin;
  out.length = c.compactification_length;
  out.nr = c.radial_points;
  out.ntheta = c.theta_nodes;
  out.ell_max_first = c.ell_max_first;
  out.ell_max_second = c.ell_max_second;
  out.modes = list(c.modes, c.mode_count);
  out.parents = list(c.parents, c.parent_count);
  out.targets = list(c.targets, c.target_count);
  out.damping = c.reduction_damping;
  out.dissipation = c.dissipation;
  out.reduction = c.reduction;
  out.disc = c.discretization;
  out.source_mode = c.source_mode;
  out.source_start_time = c.source_start_time;
  out.constraint_tolerance = c.normalized_constraint_tolerance;
  out.required_passes = c.required_consecutive_passes;
  if (out.source_mode < 0 || out.source_mode > 2) {
    throw std::invalid_argument("unsupported second-order source mode");
  }
  return out;
}

void ensure_constants_on_current_device() {
  static std::mutex mutex;
  static bool uploaded[128] = {};
  int device = 0;
  check(cudaGetDevice(&device), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(mutex);
  if (device >= 0 && device < 128 && uploaded[device]) return;
  check(upload_sbp_constants(build_sbp_constants()), "upload SBP constants");
  if (device >= 0 && device < 128) uploaded[device] = true;
}

template <class T>
struct DeviceArray {
  T* ptr = nullptr;
  size_t count = 0;
  bool owned = true;  // false: memory lent by a longer-lived owner
  // non-null: allocated from a memory pool, freed stream-ordered on this
  // stream (the stream every use of the memory is ordered on)
  cudaStream_t pool_stream = nullptr;
  DeviceArray() = default;
  DeviceArray(const DeviceArray&) = delete;
  DeviceArray& operator=(const DeviceArray&) = delete;
  DeviceArray(DeviceArray&& other) noexcept
      : ptr(other.ptr), count(other.count), owned(other.owned),
        pool_stream(other.pool_stream) {
    other.ptr = nullptr;
    other.count = 0;
    other.owned = true;
    other.pool_stream = nullptr;
  }
  DeviceArray& operator=(DeviceArray&& other) noexcept {
    if (this != &other) {
      release();
      ptr = other.ptr;
      count = other.count;
      owned = other.owned;
      pool_stream = other.pool_stream;
      other.ptr = nullptr;
      other.count = 0;
      other.owned = true;
      other.pool_stream = nullptr;
    }
    return *this;
  }
  void allocate(const size_t n) {
    release();
    if (n == 0) return;
    check(cudaMalloc(reinterpret_cast<void**>(&ptr), n * sizeof(T)),
          "cudaMalloc");
    count = n;
  }
  void allocate_from_pool(const size_t n, cudaMemPool_t pool,
                          cudaStream_t stream) {
    release();
    if (n == 0) return;
    check(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&ptr),
                                  n * sizeof(T), pool, stream),
          "cudaMallocFromPoolAsync");
    count = n;
    pool_stream = stream;
  }
  void borrow(T* p, const size_t n) {
    release();
    ptr = p;
    count = n;
    owned = false;
  }
  void release() {
    if (ptr != nullptr && owned) {
      if (pool_stream != nullptr) {
        cudaFreeAsync(ptr, pool_stream);
      } else {
        cudaFree(ptr);
      }
    }
    ptr = nullptr;
    count = 0;
    owned = true;
    pool_stream = nullptr;
  }
  ~DeviceArray() { release(); }
};

// Band buffers that outlive one batch layout: two state buffers (the live
// one and the next layout's) and the three RK slope buffers, grown on
// demand and lent to each Batch a server builds.  With a pool, growth is a
// stream-ordered pool allocation: the pool keeps freed blocks (release
// threshold: never), so a layout change does not return memory to the
// driver or wait on a device-wide free.  Capacity grows geometrically (at
// least doubling), capped at what the HBM budget lets one buffer hold.
struct StateArena {
  DeviceArray<double2> y[2];
  DeviceArray<double2> kA, kB, acc;
  int current = 0;                // y[current] holds the live batch's state
  cudaMemPool_t pool = nullptr;   // null: plain cudaMalloc
  cudaStream_t stream = nullptr;  // every use of the buffers is ordered on it
  size_t cap = ~size_t{0};        // complex values one buffer may grow to
  void grow(DeviceArray<double2>& a, const size_t n) {
    if (a.count >= n) return;
    const size_t want =
        std::max(n, std::min(std::max(n + n / 4, 2 * a.count), cap));
    if (pool != nullptr) {
      a.allocate_from_pool(want, pool, stream);
    } else {
      a.allocate(want);
    }
  }
  void release() {
    for (auto* a : {&y[0], &y[1], &kA, &kB, &acc}) a->release();
  }
};

constexpr int kTargetTileRows = 48;
constexpr int kStageRowBlock = 2;  // rows per stage-kernel work item
constexpr size_t kSmemBudget = 200 * 1024;

// Stage kernel of a band: the narrow streaming kernel (n_ell <= 16, at most
// 32 nodes), the wide one (n_ell <= 24, at most 48 nodes, free-damped) or
// the tile kernel.
constexpr int kKindNarrow = 0, kKindWide = 1, kKindTile = 2;
int stage_kernel_kind(const InstanceDesc& in, const int n_ell,
                      const bool tile_only) {
  if (tile_only) return kKindTile;
  if (n_ell <= kStreamMaxEll && in.ntheta <= kStreamMaxNodes) return kKindNarrow;
  if (n_ell <= kWideMaxEll && in.ntheta <= kWideMaxNodes && in.reduction == 0) {
    return kKindWide;
  }
  return kKindTile;
}

int slab_halo(const int disc, const int reduction) {
  const DiscInfo info = disc_info(disc);
  return reduction == 1 ? std::max(info.diss_order, 2 * info.interior_half)
                        : info.diss_order;
}

}  // namespace

struct Batch {
  std::vector<InstancePlan> plans;
  std::vector<std::vector<int>> instance_segments;  // segment ids
  std::vector<InstanceDesc> h_inst;
  std::vector<SegmentDesc> h_seg;
  std::vector<int> seg_mode;  // registry index of each segment's mode
  std::vector<TileDesc> h_tiles;
  std::vector<double> h_mat;
  std::vector<double> h_trig;
  std::vector<StageLaunch> groups;  // one per (disc, reduction)
  // Launch groups of one stage touch disjoint segments: groups after the
  // first run on these streams, forked from and joined back into `stream`
  // (inside a captured step they become parallel graph branches).
  std::vector<cudaStream_t> group_streams;
  std::vector<cudaEvent_t> group_events;  // [0] fork, [i] join of stream i
  std::vector<int> group_first_tile;
  std::vector<TileDesc> h_strips;       // streaming-kernel strips
  std::vector<int> group_first_strip;   // -1: group runs the tile kernel
  size_t total_complex = 0;
  int max_ell = 1;

  DeviceArray<double2> y, kA, kB, acc;
  DeviceArray<InstanceDesc> d_inst;
  DeviceArray<SegmentDesc> d_seg;
  DeviceArray<int> d_seg_mode;
  DeviceArray<TileDesc> d_tiles;
  DeviceArray<TileDesc> d_strips;
  DeviceArray<int> d_error;  // streaming-kernel wait timeouts
  DeviceArray<double> d_coef;  // Teukolsky row coefficients per solve row
  DeviceArray<double> d_nodes;  // 1 / C_T on the nodes per solve row
  DeviceArray<double> d_nodes_wide;  // the same, kWideMaxNodes per row
  int wide_rows = 0;  // rows of the wide node table
  int withhold_chunk_ = -1;    // failure-detection test hook
  teuk_b200_batch_options options{TEUK_B200_ABI_VERSION, TEUK_B200_KERNEL_AUTO,
                                  TEUK_B200_PRECISION_FP64, 0, 0};
  std::vector<int> group_strip_rows;  // strip length per group (0: tile)
  // strips of streaming group g live in h_strips / d_strips at
  // [group_first_strip[g], + group_strip_capacity[g]): room for the most
  // strips any strip length gives, so retuning one group moves no other
  std::vector<int> group_strip_capacity;
  std::vector<std::vector<int>> group_segments_;  // segments of each group
  int coef_rows = 0;
  DeviceArray<double> d_mat, d_trig;
  // split-precision digit records of every segment (streaming kernel)
  std::vector<uint4> h_split;
  std::vector<double> h_split_scale;
  DeviceArray<uint4> d_split;
  DeviceArray<double> d_split_scale;
  DeviceArray<double2> d_nodal;     // one instance's nodal state (lazy)
  size_t nodal_max = 0;
  DeviceArray<double2> d_endpoint;  // gathered endpoint coefficients
  DeviceArray<int> d_parent_mask;    // per instance, per registry mode
  DeviceArray<int> d_flag;
  std::vector<size_t> parent_mask_offset;
  std::vector<DeviceArray<double2>> frozen_dev;  // per instance, or empty

  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  // a server's memory pool and stream (null: cudaMalloc): where the
  // batch's device buffers come from
  cudaMemPool_t pool = nullptr;
  cudaStream_t pool_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;
  bool dt_dirty = false;

  ~Batch() {
    if (graph_exec != nullptr) cudaGraphExecDestroy(graph_exec);
    if (graph != nullptr) cudaGraphDestroy(graph);
    for (cudaStream_t s : group_streams) cudaStreamDestroy(s);
    for (cudaEvent_t e : group_events) cudaEventDestroy(e);
    if (own_stream != nullptr) cudaStreamDestroy(own_stream);
  }

  void build(const std::vector<Config>& configs) {
    if (configs.empty()) {
      throw std::invalid_argument("a batch needs at least one solve");
    }
    std::vector<InstancePlan> planned;
    for (const Config& c : configs) {
      // The reference's construction-time validation runs first, so invalid
      // inputs report the same error whatever their source policy.
      planned.push_back(build_instance_plan(c));
    }
    build_planned(std::move(planned));
  }

  double2* nodal_scratch() {
    if (d_nodal.ptr == nullptr) alloc(d_nodal, nodal_max);
    return d_nodal.ptr;
  }

  // A device buffer of this batch: from the server's pool (stream-ordered
  // on the server's stream, the stream this batch runs on) or cudaMalloc.
  template <class T>
  void alloc(DeviceArray<T>& a, const size_t n) {
    if (pool != nullptr) {
      a.allocate_from_pool(n, pool, pool_stream);
    } else {
      a.allocate(n);
    }
  }

  // Layout and device buffers for already validated plans.  With an arena
  // the band buffers are borrowed from it (the state buffer that is not
  // live) instead of allocated.
  void build_planned(std::vector<InstancePlan> planned,
                     StateArena* arena = nullptr) {
    if (planned.empty()) {
      throw std::invalid_argument("a batch needs at least one solve");
    }
    plans = std::move(planned);
    for (const InstancePlan& plan : plans) {
      const Config& c = plan.config;
      if (c.source_mode != 0) {
        throw Unsupported(
            "second-order source policies run through teuk_b200_create "
            "(one nodal pipeline per solve), not through a batch");
      }
    }
    int device_count = 0;
    check(cudaGetDeviceCount(&device_count), "cudaGetDeviceCount");
    if (device_count <= 0) throw CudaError("no CUDA device is visible");
    ensure_constants_on_current_device();

    // Segments, matrices, trig tables.
    long long offset = 0;
    for (size_t i = 0; i < plans.size(); ++i) {
      InstancePlan& plan = plans[i];
      const Config& c = plan.config;
      InstanceDesc d{};
      d.mass = c.mass;
      d.spin = c.spin;
      d.length = c.length;
      d.spacing = plan.spacing;
      d.inv_spacing = 1.0 / plan.spacing;
      d.damping = c.reduction == 0 ? c.damping : 0.0;
      d.dissipation = c.dissipation;
      d.dt = 0.0;
      d.nr = c.nr;
      d.ntheta = c.ntheta;
      d.trig_offset = static_cast<int>(h_trig.size());
      d.reduction = c.reduction;
      d.disc = c.disc;
      d.coef_row0 = coef_rows;
      coef_rows += c.nr;
      h_trig.insert(h_trig.end(), plan.sinv.begin(), plan.sinv.end());
      h_trig.insert(h_trig.end(), plan.cosv.begin(), plan.cosv.end());
      h_inst.push_back(d);
      instance_segments.emplace_back();
      for (ModePlan& mp : plan.modes) {
        if (!mp.parent) continue;
        SegmentDesc s{};
        s.offset = offset;
        s.instance = static_cast<int>(i);
        s.m = mp.m;
        s.n_ell = mp.n_ell;
        s.ell_min = mp.ell_min;
        s.row_stride = 3 * mp.n_ell;
        s.mat_offset = static_cast<int>(h_mat.size());
        const int ne = mp.n_ell, nt = c.ntheta;
        // St[l][j] then At[j][l]
        for (int l = 0; l < ne; ++l) {
          for (int j = 0; j < nt; ++j) {
            h_mat.push_back(mp.synthesis[static_cast<size_t>(j) * ne + l]);
          }
        }
        for (int j = 0; j < nt; ++j) {
          for (int l = 0; l < ne; ++l) {
            h_mat.push_back(mp.analysis[static_cast<size_t>(l) * nt + j]);
          }
        }
        append_split_record(mp, nt);
        mp.segment = static_cast<long long>(h_seg.size());
        instance_segments.back().push_back(static_cast<int>(h_seg.size()));
        h_seg.push_back(s);
        seg_mode.push_back(mp.mode_index);
        max_ell = std::max(max_ell, ne);
        long long count = static_cast<long long>(c.nr) * 3 * ne;
        count = (count + 15) / 16 * 16;  // 256-byte aligned segments
        offset += count;
      }
    }
    total_complex = static_cast<size_t>(offset);

    // Launch groups by (disc, reduction) and stage kernel: segments with
    // n_ell <= 16 of solves with at most 32 nodes run the streaming kernel
    // (radial strips), the others the tile kernel (radial tiles).  Segments
    // do not couple, so a solve may have segments in both.
    const bool tile_only = options.stage_kernel == TEUK_B200_KERNEL_TILE;
    withhold_chunk_ = g_test_withhold_chunk.load();
    const auto kind_of = [&](const size_t s) {
      return stage_kernel_kind(h_inst[static_cast<size_t>(h_seg[s].instance)],
                               h_seg[s].n_ell, tile_only);
    };
    // rows of the wide node table: solves with bands on the wide kernel
    wide_rows = 0;
    for (size_t i = 0; i < h_inst.size(); ++i) {
      bool wide = false;
      for (const int s : instance_segments[i]) {
        wide = wide || kind_of(static_cast<size_t>(s)) == kKindWide;
      }
      h_inst[i].wide_row0 = wide ? wide_rows : -1;
      if (wide) wide_rows += h_inst[i].nr;
    }
    for (int disc = 0; disc < 3; ++disc) {
      for (int red = 0; red < 2; ++red) {
       for (int kind = 0; kind < 3; ++kind) {  // narrow, wide, tile kernel
        StageLaunch g{};
        g.disc = disc;
        g.reduction = red;
        const int first_tile = static_cast<int>(h_tiles.size());
        const int H = slab_halo(disc, red);
        const int HD = disc_info(disc).interior_half;
        std::vector<int> group_segments;
        for (size_t s = 0; s < h_seg.size(); ++s) {
          const InstanceDesc& in = h_inst[static_cast<size_t>(h_seg[s].instance)];
          if (in.disc != disc || in.reduction != red) continue;
          if (kind_of(s) != kind) continue;
          group_segments.push_back(static_cast<int>(s));
          const int ne = h_seg[s].n_ell;
          const int nr = in.nr;
          // at most one (row pair, ell) work item per thread, so the stage
          // kernel can park its results and stream the RK update
          int rows = std::min(kTargetTileRows,
                              std::max(16, (256 / ne) * kStageRowBlock));
          int tiles = (nr + rows - 1) / rows;
          tiles = std::max(1, std::min(tiles, nr / 16));
          for (int t = 0; t < tiles; ++t) {
            const int r0 = static_cast<int>(static_cast<long long>(nr) * t / tiles);
            const int r1 =
                static_cast<int>(static_cast<long long>(nr) * (t + 1) / tiles);
            h_tiles.push_back({static_cast<int>(s), r0, r1, 0});
            const int s0 = std::max(0, r0 - H), s1 = std::min(nr, r1 + H);
            const int t0 = std::max(0, r0 - HD), t1 = std::min(nr, r1 + HD);
            g.slab_capacity = std::max(g.slab_capacity, (s1 - s0) * 3 * ne);
            g.dslab_capacity = std::max(g.dslab_capacity, (t1 - t0) * ne);
            g.coef_rows = std::max(g.coef_rows, t1 - t0);
          }
          g.matrix_capacity =
              std::max(g.matrix_capacity, ne * in.ntheta);
          g.max_theta = std::max(g.max_theta, in.ntheta);
          g.max_ell = std::max(g.max_ell, ne);
        }
        g.tile_count = static_cast<int>(h_tiles.size()) - first_tile;
        if (g.tile_count > 0) {
          if (kind == kKindTile && stage_smem_bytes(g) > kSmemBudget) {
            throw std::invalid_argument(
                "solve shape exceeds the stage kernel's shared-memory tile");
          }
          g.strips = nullptr;
          g.strip_count = 0;
          g.wide = kind == kKindWide ? 1 : 0;
          if (kind != kKindTile) {
            plan_strip_region(g, group_segments);
          } else {
            group_first_strip.push_back(-1);
            group_strip_capacity.push_back(0);
            group_strip_rows.push_back(0);
            group_segments_.push_back({});
          }
          groups.push_back(g);
          group_first_tile.push_back(first_tile);
        }
       }
      }
    }

    // Device allocations: from the server's memory pool when a server
    // builds the batch (no driver allocation or device-wide free on a
    // layout change), plain cudaMalloc otherwise.
    if (arena != nullptr && arena->pool != nullptr) {
      pool = arena->pool;
      pool_stream = arena->stream;
    }
    if (arena != nullptr) {
      DeviceArray<double2>& next = arena->y[1 - arena->current];
      arena->grow(next, total_complex);
      arena->grow(arena->kA, total_complex);
      arena->grow(arena->kB, total_complex);
      arena->grow(arena->acc, total_complex);
      y.borrow(next.ptr, total_complex);
      kA.borrow(arena->kA.ptr, total_complex);
      kB.borrow(arena->kB.ptr, total_complex);
      acc.borrow(arena->acc.ptr, total_complex);
    } else {
      y.allocate(total_complex);
      kA.allocate(total_complex);
      kB.allocate(total_complex);
      acc.allocate(total_complex);
    }
    nodal_max = 0;
    for (const InstancePlan& plan : plans) {
      nodal_max = std::max(nodal_max, plan.value_count());
    }
    std::vector<int> mask;
    for (const InstancePlan& plan : plans) {
      parent_mask_offset.push_back(mask.size());
      for (const ModePlan& mp : plan.modes) mask.push_back(mp.parent ? 1 : 0);
    }
    alloc(d_inst, h_inst.size());
    alloc(d_seg, h_seg.size());
    alloc(d_seg_mode, seg_mode.size());
    alloc(d_tiles, h_tiles.size());
    alloc(d_strips, std::max<size_t>(h_strips.size(), 1));
    alloc(d_error, 1);
    alloc(d_coef, static_cast<size_t>(std::max(coef_rows, 1)) * kCoefRecord);
    alloc(d_nodes, static_cast<size_t>(std::max(coef_rows, 1)) * kNodeRecord);
    alloc(d_nodes_wide, static_cast<size_t>(std::max(wide_rows, 1)) * kWideMaxNodes);
    alloc(d_mat, std::max<size_t>(h_mat.size(), 1));
    alloc(d_split, std::max<size_t>(h_split.size(), 1));
    alloc(d_split_scale, std::max<size_t>(h_split_scale.size(), 1));
    alloc(d_trig, h_trig.size());
    alloc(d_endpoint,
          std::max<size_t>(h_seg.size(), 1) * 2 * static_cast<size_t>(max_ell));
    alloc(d_parent_mask, mask.size());
    alloc(d_flag, 1);
    // pool memory is usable from every stream once the allocating stream
    // has been reached
    if (pool != nullptr) check(cudaStreamSynchronize(pool_stream), "pool allocations");
    check(cudaMemset(y.ptr, 0, total_complex * sizeof(double2)), "memset y");
    check(cudaMemset(d_error.ptr, 0, sizeof(int)), "memset error word");
    check(cudaMemcpy(d_parent_mask.ptr, mask.data(), mask.size() * sizeof(int),
                     cudaMemcpyHostToDevice),
          "upload parent mask");
    frozen_dev.resize(plans.size());
    check(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking),
          "cudaStreamCreate");
    stream = own_stream;
    upload_descriptors();
    check(cudaMemcpy(d_seg.ptr, h_seg.data(), h_seg.size() * sizeof(SegmentDesc),
                     cudaMemcpyHostToDevice),
          "upload segments");
    check(cudaMemcpy(d_seg_mode.ptr, seg_mode.data(),
                     seg_mode.size() * sizeof(int), cudaMemcpyHostToDevice),
          "upload segment modes");
    check(cudaMemcpy(d_tiles.ptr, h_tiles.data(),
                     h_tiles.size() * sizeof(TileDesc), cudaMemcpyHostToDevice),
          "upload tiles");
    if (!h_strips.empty()) {
      check(cudaMemcpy(d_strips.ptr, h_strips.data(),
                       h_strips.size() * sizeof(TileDesc),
                       cudaMemcpyHostToDevice),
            "upload strips");
    }
    if (!h_mat.empty()) {
      check(cudaMemcpy(d_mat.ptr, h_mat.data(), h_mat.size() * sizeof(double),
                       cudaMemcpyHostToDevice),
            "upload matrices");
    }
    if (!h_split.empty()) {
      check(cudaMemcpy(d_split.ptr, h_split.data(), h_split.size() * sizeof(uint4),
                       cudaMemcpyHostToDevice),
            "upload split records");
      check(cudaMemcpy(d_split_scale.ptr, h_split_scale.data(),
                       h_split_scale.size() * sizeof(double),
                       cudaMemcpyHostToDevice),
            "upload split scales");
    }
    check(cudaMemcpy(d_trig.ptr, h_trig.data(), h_trig.size() * sizeof(double),
                     cudaMemcpyHostToDevice),
          "upload trig");
    for (size_t i = 0; i < h_inst.size(); ++i) {
      check(launch_coefficient_table(d_inst.ptr + i, d_trig.ptr, h_inst[i].nr,
                                     h_inst[i].coef_row0, d_coef.ptr,
                                     d_nodes.ptr, h_inst[i].coef_row0,
                                     kNodeRecord, stream),
            "coefficient table");
      if (h_inst[i].wide_row0 >= 0) {  // node rows only
        check(launch_coefficient_table(d_inst.ptr + i, d_trig.ptr, h_inst[i].nr,
                                       0, nullptr, d_nodes_wide.ptr,
                                       h_inst[i].wide_row0, kWideMaxNodes,
                                       stream),
              "wide node table");
      }
    }
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      StageLaunch& g = groups[gi];
      g.tiles = d_tiles.ptr + group_first_tile[gi];
      g.error = d_error.ptr;
      g.coef_table = d_coef.ptr;
      g.node_table = g.wide ? d_nodes_wide.ptr : d_nodes.ptr;
      g.withhold_chunk = withhold_chunk_;
      // the wide kernel and the tile kernel transform in FP64
      g.precision =
          options.precision == TEUK_B200_PRECISION_SPLIT && !g.wide ? 1 : 0;
      g.split_frags = d_split.ptr;
      g.split_scales = d_split_scale.ptr;
      if (group_first_strip[gi] >= 0) {
        g.strips = d_strips.ptr + group_first_strip[gi];
      } else {
        g.strips = nullptr;
        g.strip_count = 0;
      }
      g.instances = d_inst.ptr;
      g.segments = d_seg.ptr;
      g.matrices = d_mat.ptr;
      g.trig = d_trig.ptr;
      g.y = y.ptr;
      g.kA = kA.ptr;
      g.kB = kB.ptr;
      g.acc = acc.ptr;
    }
    if (options.autotune != 0 && options.strip_rows == 0) autotune_strips();
  }

  // Split-precision digit record of one segment for the streaming kernel's
  // transforms: BF16 digit fragments of the synthesis matrix S(j, l) (rows =
  // nodes, one power-of-two scale per node) and of the analysis matrix
  // A(l, j) (rows = ell, one scale per ell), in the m16n8k16 A-operand
  // layout of the two transform warps, [synthesis h0, h1, analysis h0,
  // h1][slice][lane]; then 32 node scales and 16 ell scales 2^(F - 14).
  // Segments outside the streaming kernel's shapes get a zero record.
  void append_split_record(const ModePlan& mp, const int nt) {
    namespace sp = teuk_b200::split;
    const int ne = mp.n_ell;
    const bool fits = ne <= kStreamMaxEll && nt <= kStreamMaxNodes;
    const size_t base = h_split.size();
    h_split.resize(base + kSplitRecordUint4, uint4{0u, 0u, 0u, 0u});
    const size_t sbase = h_split_scale.size();
    h_split_scale.resize(sbase + kSplitScaleDoubles, 0.0);
    if (!fits) return;
    const auto S = [&](const int j, const int l) {
      return (j < nt && l < ne) ? mp.synthesis[static_cast<size_t>(j) * ne + l] : 0.0;
    };
    const auto A = [&](const int l, const int j) {
      return (j < nt && l < ne) ? mp.analysis[static_cast<size_t>(l) * nt + j] : 0.0;
    };
    // digits[row][k][slice] of the row-scaled matrices (16 x 32 / 32 x 16)
    float ds[kStreamMaxNodes][kStreamMaxEll][sp::kSlices] = {};
    float da[kStreamMaxEll][kStreamMaxNodes][sp::kSlices] = {};
    for (int j = 0; j < kStreamMaxNodes; ++j) {
      double m = 0.0;
      for (int l = 0; l < kStreamMaxEll; ++l) m = std::max(m, std::fabs(S(j, l)));
      const int e = sp::host_exponent(m);
      h_split_scale[sbase + j] = std::ldexp(1.0, e - 14);
      for (int l = 0; l < kStreamMaxEll; ++l) {
        sp::host_digits(S(j, l) * std::ldexp(1.0, -e), ds[j][l]);
      }
    }
    for (int l = 0; l < kStreamMaxEll; ++l) {
      double m = 0.0;
      for (int j = 0; j < kStreamMaxNodes; ++j) m = std::max(m, std::fabs(A(l, j)));
      const int e = sp::host_exponent(m);
      h_split_scale[sbase + kStreamMaxNodes + l] = std::ldexp(1.0, e - 14);
      for (int j = 0; j < kStreamMaxNodes; ++j) {
        sp::host_digits(A(l, j) * std::ldexp(1.0, -e), da[l][j]);
      }
    }
    for (int h = 0; h < 2; ++h) {
      for (int sl = 0; sl < sp::kSlices; ++sl) {
        for (int lane = 0; lane < 32; ++lane) {
          const int g = lane / 4, q = lane % 4;
          // synthesis: rows nodes 16h + g (+8), k = ell
          const int j0 = 16 * h + g, j1 = j0 + 8;
          uint4 f;
          f.x = sp::host_pack(ds[j0][2 * q][sl], ds[j0][2 * q + 1][sl]);
          f.y = sp::host_pack(ds[j1][2 * q][sl], ds[j1][2 * q + 1][sl]);
          f.z = sp::host_pack(ds[j0][2 * q + 8][sl], ds[j0][2 * q + 9][sl]);
          f.w = sp::host_pack(ds[j1][2 * q + 8][sl], ds[j1][2 * q + 9][sl]);
          h_split[base + (h * sp::kSlices + sl) * 32 + lane] = f;
          // analysis: rows ell g (+8), k = nodes 16h + 2q (+1, +8, +9)
          const int k0 = 16 * h + 2 * q;
          uint4 a;
          a.x = sp::host_pack(da[g][k0][sl], da[g][k0 + 1][sl]);
          a.y = sp::host_pack(da[g + 8][k0][sl], da[g + 8][k0 + 1][sl]);
          a.z = sp::host_pack(da[g][k0 + 8][sl], da[g][k0 + 9][sl]);
          a.w = sp::host_pack(da[g + 8][k0 + 8][sl], da[g + 8][k0 + 9][sl]);
          h_split[base + ((2 + h) * sp::kSlices + sl) * 32 + lane] = a;
        }
      }
    }
  }

  // Radial strips of a streaming launch group (its segments `segs`) for a
  // strip length of `target` rows, sorted by n_ell (largest first) so that
  // a CTA's consecutive strips mostly share one ring row stride.  A segment
  // of nr rows becomes max(1, min(nr / target, nr / 64)) balanced strips.
  std::vector<TileDesc> make_strips(std::vector<int> segs, const int target) const {
    std::stable_sort(segs.begin(), segs.end(), [&](const int a, const int b) {
      return h_seg[static_cast<size_t>(a)].n_ell > h_seg[static_cast<size_t>(b)].n_ell;
    });
    std::vector<TileDesc> out;
    for (const int s : segs) {
      const int nr = h_inst[static_cast<size_t>(h_seg[static_cast<size_t>(s)].instance)].nr;
      int n = std::max(1, nr / target);
      n = std::max(1, std::min(n, nr / kStripMinRows));
      for (int t = 0; t < n; ++t) {
        const int r0 = static_cast<int>(static_cast<long long>(nr) * t / n);
        const int r1 = static_cast<int>(static_cast<long long>(nr) * (t + 1) / n);
        out.push_back({s, r0, r1, 0});
      }
    }
    return out;
  }

  // Built-in strip length: about kStripsPerCta strips per SM over the
  // group's rows, between 64 and 1024 rows.
  static int default_strip_rows(const long long rows, const int sms) {
    const long long want = static_cast<long long>(std::max(sms, 1)) * kStripsPerCta;
    return static_cast<int>(std::min<long long>(
        1024, std::max<long long>(kStripMinRows, rows / want)));
  }

  long long group_rows(const std::vector<int>& segs) const {
    long long rows = 0;
    for (const int s : segs) {
      rows += h_inst[static_cast<size_t>(h_seg[static_cast<size_t>(s)].instance)].nr;
    }
    return rows;
  }

  int device_sms() const {
    int device = 0, sms = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device),
          "SM count");
    return sms;
  }

  // Reserves the strip region of a new streaming group and fills it with
  // the strips of the requested (or built-in) strip length.
  void plan_strip_region(StageLaunch& g, const std::vector<int>& segs) {
    const int max_ell = g.wide ? kWideMaxEll : kStreamMaxEll;
    const int max_theta = g.wide ? kWideMaxNodes : kStreamMaxNodes;
    if (g.max_ell > max_ell || g.max_theta > max_theta ||
        (g.wide && g.reduction != 0)) {
      throw std::logic_error("segment outside the streaming kernel's shapes");
    }
    const int target = options.strip_rows > 0
                           ? options.strip_rows
                           : default_strip_rows(group_rows(segs), device_sms());
    const int first = static_cast<int>(h_strips.size());
    const int capacity = static_cast<int>(make_strips(segs, kStripMinRows).size());
    std::vector<TileDesc> strips = make_strips(segs, target);
    h_strips.insert(h_strips.end(), strips.begin(), strips.end());
    h_strips.resize(static_cast<size_t>(first + capacity), TileDesc{0, 0, 0, 0});
    g.strip_count = static_cast<int>(strips.size());
    group_first_strip.push_back(first);
    group_strip_capacity.push_back(capacity);
    group_strip_rows.push_back(target);
    group_segments_.push_back(segs);
  }

  // Writes strips into group gi's region of the device strip table.
  void upload_group_strips(const size_t gi, const std::vector<TileDesc>& strips) {
    std::copy(strips.begin(), strips.end(),
              h_strips.begin() + group_first_strip[gi]);
    check(cudaMemcpyAsync(d_strips.ptr + group_first_strip[gi], strips.data(),
                          strips.size() * sizeof(TileDesc),
                          cudaMemcpyHostToDevice, stream),
          "upload strips");
    groups[gi].strip_count = static_cast<int>(strips.size());
  }

  // The strip-length autotuner.  For every streaming launch group it times
  // one RK4 step (the four stage launches) of the group for each candidate
  // strip length (64 to 4096 rows, up to the longest segment) and keeps the
  // fastest; the choice is cached for the
  // process by (kernel, discretization, reduction, widest band, rows
  // rounded to a quarter octave, SM count).  Strips only decide which CTA streams which
  // rows: every row gets the same sums in the same order for any choice,
  // so results are bit-identical across choices.  Runs at build, on the
  // zero state (every stage of a zero state is zero, and stages 2-4 read
  // only what the stages before them wrote).
  void autotune_strips() {
    static std::mutex cache_mutex;
    static std::map<std::tuple<int, int, int, int, int, int>, int> cache;
    static const int kCandidates[] = {64,  96,  128,  192,  256,  384,
                                      512, 768, 1024, 1536, 2048, 4096};
    const int sms = device_sms();
    cudaEvent_t ev[2] = {nullptr, nullptr};
    for (cudaEvent_t& e : ev) check(cudaEventCreate(&e), "cudaEventCreate");
    for (size_t gi = 0; gi < groups.size(); ++gi) {
      if (group_first_strip[gi] < 0) continue;
      const auto& segs = group_segments_[gi];
      const long long rows = group_rows(segs);
      int max_nr = 0;
      for (const int s : segs) {
        max_nr = std::max(max_nr, h_inst[static_cast<size_t>(h_seg[static_cast<size_t>(s)].instance)].nr);
      }
      const auto key = std::make_tuple(
          groups[gi].wide, groups[gi].disc, groups[gi].reduction, groups[gi].max_ell,
          static_cast<int>(std::lround(4.0 * std::log2(static_cast<double>(rows)))),
          sms);
      int best = -1;
      {
        std::lock_guard<std::mutex> lock(cache_mutex);
        const auto it = cache.find(key);
        if (it != cache.end()) best = it->second;
      }
      if (best < 0) {
        float best_ms = std::numeric_limits<float>::infinity();
        for (const int c : kCandidates) {
          if (c > std::max(max_nr, kStripMinRows)) break;
          upload_group_strips(gi, make_strips(segs, c));
          float ms = std::numeric_limits<float>::infinity();
          for (int rep = 0; rep < 3; ++rep) {
            check(cudaEventRecord(ev[0], stream), "event");
            for (int kind = kStage1; kind <= kStage4; ++kind) {
              StageLaunch g = groups[gi];
              g.stage = kind;
              check(launch_stage(g, stream), "stage kernel");
            }
            check(cudaEventRecord(ev[1], stream), "event");
            check(cudaEventSynchronize(ev[1]), "autotune step");
            float t = 0.0f;
            check(cudaEventElapsedTime(&t, ev[0], ev[1]), "event time");
            if (rep > 0) ms = std::min(ms, t);
          }
          if (ms < best_ms) {
            best_ms = ms;
            best = c;
          }
        }
        std::lock_guard<std::mutex> lock(cache_mutex);
        cache[key] = best;
      }
      upload_group_strips(gi, make_strips(segs, best));
      group_strip_rows[gi] = best;
    }
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    check(cudaStreamSynchronize(stream), "autotune");
    check_kernel_error();
    // the stages ran on the zero state: y is still zero, the slopes are
    // rewritten by the first step
  }

  // Raises the error a streaming-kernel wait recorded (after a stream sync).
  void check_kernel_error() {
    if (d_error.ptr == nullptr) return;
    int code = 0;
    check(cudaMemcpy(&code, d_error.ptr, sizeof(int), cudaMemcpyDeviceToHost),
          "read kernel error word");
    if (code != 0) {
      cudaMemset(d_error.ptr, 0, sizeof(int));
      throw CudaError("stage kernel pipeline wait timed out (code " +
                      std::to_string(code) + ")");
    }
  }

  void upload_descriptors() {
    check(cudaMemcpyAsync(d_inst.ptr, h_inst.data(),
                          h_inst.size() * sizeof(InstanceDesc),
                          cudaMemcpyHostToDevice, stream),
          "upload instances");
    dt_dirty = false;
  }

  void check_instance(const int instance) const {
    if (instance < 0 || instance >= static_cast<int>(plans.size())) {
      throw std::out_of_range("batch instance index is out of range");
    }
  }

  ConvertLaunch convert(const int instance) {
    const InstancePlan& plan = plans[static_cast<size_t>(instance)];
    ConvertLaunch c{};
    c.modal = y.ptr;
    const auto& segs = instance_segments[static_cast<size_t>(instance)];
    c.segments = d_seg.ptr + (segs.empty() ? 0 : segs.front());
    c.segment_modes = d_seg_mode.ptr + (segs.empty() ? 0 : segs.front());
    c.matrices = d_mat.ptr;
    c.segment_count = static_cast<int>(segs.size());
    c.nr = plan.config.nr;
    c.ntheta = plan.config.ntheta;
    c.mode_count = static_cast<int>(plan.config.modes.size());
    c.max_ell = max_ell;
    return c;
  }

  void set_state(const int instance, const double* state, const size_t count,
                 const int memory) {
    check_instance(instance);
    InstancePlan& plan = plans[static_cast<size_t>(instance)];
    if (count != plan.value_count()) {
      throw std::invalid_argument("state complex count does not match shape");
    }
    if (state == nullptr) throw std::invalid_argument("null state pointer");
    const size_t bytes = count * sizeof(double2);
    const double2* source = nullptr;
    if (memory == TEUK_B200_HOST) {
      check(cudaMemcpyAsync(nodal_scratch(), state, bytes, cudaMemcpyHostToDevice,
                            stream),
            "set_state upload");
      source = nodal_scratch();
    } else if (memory == TEUK_B200_DEVICE) {
      source = reinterpret_cast<const double2*>(state);
    } else {
      throw std::invalid_argument("unknown memory kind");
    }
    // Frozen planes (every field of a non-parent mode, fields 3..12 of a
    // parent) never change in the linear pipeline; a device copy is kept
    // only when one of them is non-zero.
    check(cudaMemsetAsync(d_flag.ptr, 0, sizeof(int), stream), "flag reset");
    check(launch_frozen_scan(source,
                             d_parent_mask.ptr + parent_mask_offset[static_cast<size_t>(instance)],
                             static_cast<int>(plan.config.modes.size()),
                             plan.config.nr * plan.config.ntheta, d_flag.ptr,
                             stream),
          "frozen scan");
    ConvertLaunch c = convert(instance);
    c.nodal_in = source;
    check(launch_nodal_to_modal(c, stream), "nodal_to_modal");
    int flag = 0;
    check(cudaMemcpyAsync(&flag, d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost,
                          stream),
          "flag read");
    check(cudaStreamSynchronize(stream), "set_state");
    auto& frozen = frozen_dev[static_cast<size_t>(instance)];
    if (flag != 0) {
      if (frozen.count != count) alloc(frozen, count);
      check(cudaMemcpyAsync(frozen.ptr, source, bytes, cudaMemcpyDeviceToDevice,
                            stream),
            "frozen copy");
      check(cudaStreamSynchronize(stream), "frozen copy");
    } else {
      frozen.release();
    }
  }

  // Full nodal state of `instance` into d_nodal: frozen planes from the
  // device copy (zero when none is kept), evolved fields synthesized from
  // `modal`.
  void assemble_nodal(const int instance, double2* modal, const bool zero_frozen) {
    InstancePlan& plan = plans[static_cast<size_t>(instance)];
    const size_t bytes = plan.value_count() * sizeof(double2);
    const auto& frozen = frozen_dev[static_cast<size_t>(instance)];
    if (zero_frozen || frozen.ptr == nullptr) {
      check(cudaMemsetAsync(nodal_scratch(), 0, bytes, stream), "zero nodal");
    } else {
      check(cudaMemcpyAsync(nodal_scratch(), frozen.ptr, bytes,
                            cudaMemcpyDeviceToDevice, stream),
            "frozen restore");
    }
    ConvertLaunch c = convert(instance);
    c.modal = modal;
    c.nodal_out = nodal_scratch();
    check(launch_modal_to_nodal(c, stream), "modal_to_nodal");
  }

  void get_state(const int instance, double* out, const size_t count,
                 const int memory) {
    check_instance(instance);
    InstancePlan& plan = plans[static_cast<size_t>(instance)];
    if (count != plan.value_count()) {
      throw std::invalid_argument("state complex count does not match shape");
    }
    if (out == nullptr) throw std::invalid_argument("null state pointer");
    assemble_nodal(instance, y.ptr, false);
    const size_t bytes = count * sizeof(double2);
    check(cudaMemcpyAsync(out, nodal_scratch(), bytes,
                          memory == TEUK_B200_HOST ? cudaMemcpyDeviceToHost
                                                   : cudaMemcpyDeviceToDevice,
                          stream),
          "get_state copy");
    check(cudaStreamSynchronize(stream), "get_state");
    check_kernel_error();
  }

  void launch_stage_kind(const int kind, double2* input) {
    if (groups.size() <= 1) {
      for (StageLaunch g : groups) {
        g.stage = kind;
        if (input != nullptr) g.y = input;
        check(launch_stage(g, stream), "stage kernel");
      }
      return;
    }
    while (group_streams.size() + 1 < groups.size()) {
      cudaStream_t s = nullptr;
      check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking),
            "cudaStreamCreate");
      group_streams.push_back(s);
    }
    while (group_events.size() < groups.size()) {
      cudaEvent_t e = nullptr;
      check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming),
            "cudaEventCreate");
      group_events.push_back(e);
    }
    check(cudaEventRecord(group_events[0], stream), "fork");
    for (size_t i = 0; i < groups.size(); ++i) {
      StageLaunch g = groups[i];
      g.stage = kind;
      if (input != nullptr) g.y = input;
      cudaStream_t s = i == 0 ? stream : group_streams[i - 1];
      if (i > 0) check(cudaStreamWaitEvent(s, group_events[0], 0), "fork");
      check(launch_stage(g, s), "stage kernel");
      if (i > 0) {
        check(cudaEventRecord(group_events[i], s), "join");
        check(cudaStreamWaitEvent(stream, group_events[i], 0), "join");
      }
    }
  }

  void evaluate_rhs(const int instance, const double* stage, double* out,
                    const size_t count, const int memory) {
    check_instance(instance);
    if (plans.size() != 1) {
      throw std::invalid_argument("evaluate_rhs needs a single-solve pipeline");
    }
    InstancePlan& plan = plans[static_cast<size_t>(instance)];
    if (count != plan.value_count()) {
      throw std::invalid_argument("state complex count does not match shape");
    }
    const size_t bytes = count * sizeof(double2);
    const double2* source = reinterpret_cast<const double2*>(stage);
    if (memory == TEUK_B200_HOST) {
      check(cudaMemcpyAsync(nodal_scratch(), stage, bytes, cudaMemcpyHostToDevice,
                            stream),
            "evaluate_rhs upload");
      source = nodal_scratch();
    }
    ConvertLaunch c = convert(instance);
    c.nodal_in = source;
    c.modal = kB.ptr;
    check(launch_nodal_to_modal(c, stream), "nodal_to_modal");
    launch_stage_kind(kRhsOnly, kB.ptr);
    assemble_nodal(instance, kA.ptr, true);
    check(cudaMemcpyAsync(out, nodal_scratch(), bytes,
                          memory == TEUK_B200_HOST ? cudaMemcpyDeviceToHost
                                                   : cudaMemcpyDeviceToDevice,
                          stream),
          "evaluate_rhs copy");
    check(cudaStreamSynchronize(stream), "evaluate_rhs");
    check_kernel_error();
  }

  void set_dt(const std::vector<double>& dt) {
    for (size_t i = 0; i < h_inst.size(); ++i) {
      if (!std::isfinite(dt[i]) || !(dt[i] > 0.0)) {
        throw std::invalid_argument(
            "pipeline step requires finite positive time data");
      }
      if (h_inst[i].dt != dt[i]) {
        h_inst[i].dt = dt[i];
        dt_dirty = true;
      }
    }
    if (dt_dirty) upload_descriptors();
  }

  void record_step() {
    launch_stage_kind(kStage1, nullptr);
    launch_stage_kind(kStage2, nullptr);
    launch_stage_kind(kStage3, nullptr);
    launch_stage_kind(kStage4, nullptr);
  }

  void step(const std::vector<double>& dt, const int steps, const bool use_graph) {
    if (steps < 0) throw std::invalid_argument("step count must be nonnegative");
    set_dt(dt);
    if (!use_graph) {
      for (int s = 0; s < steps; ++s) record_step();
      check(cudaGetLastError(), "step");
      return;
    }
    if (graph_exec == nullptr || graph_stream != stream) {
      if (graph_exec != nullptr) cudaGraphExecDestroy(graph_exec);
      if (graph != nullptr) cudaGraphDestroy(graph);
      graph_exec = nullptr;
      graph = nullptr;
      check(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal),
            "begin capture");
      try {
        record_step();
      } catch (...) {
        cudaGraph_t discard = nullptr;
        cudaStreamEndCapture(stream, &discard);
        if (discard != nullptr) cudaGraphDestroy(discard);
        throw;
      }
      check(cudaStreamEndCapture(stream, &graph), "end capture");
      check(cudaGraphInstantiate(&graph_exec, graph, 0), "graph instantiate");
      graph_stream = stream;
    }
    for (int s = 0; s < steps; ++s) {
      check(cudaGraphLaunch(graph_exec, stream), "graph launch");
    }
  }

  // Gaussian initial data of one solve computed on the device straight into
  // its band segments (initialize_compactified_gaussian_pulse,
  // include/teuk/pipeline_initial_data.hpp:211-339); its frozen fields are
  // zero.
  void gaussian_device(const int instance, const double center,
                       const double width, const bool compact,
                       const std::vector<int>& ell, const std::vector<int>& m,
                       const std::vector<double>& re,
                       const std::vector<double>& im) {
    check_instance(instance);
    const InstancePlan& plan = plans[static_cast<size_t>(instance)];
    const Config& c = plan.config;
    validate_gaussian(plan, center, width, ell, m);
    const auto& segs = instance_segments[static_cast<size_t>(instance)];
    if (segs.empty()) return;
    const int nr = c.nr;
    std::vector<double> line(2 * static_cast<size_t>(nr), 0.0);
    std::vector<double> dline(2 * static_cast<size_t>(nr), 0.0);
    for (int r = 0; r < nr; ++r) {
      line[2 * static_cast<size_t>(r)] = gaussian_profile(
          plan.spacing * static_cast<double>(r), center, width, compact);
    }
    sbp_derivative_line(c.disc, line.data(), nr, 1.0 / plan.spacing,
                        dline.data());
    std::vector<double> profile(2 * static_cast<size_t>(nr));
    for (int r = 0; r < nr; ++r) {
      profile[static_cast<size_t>(r)] = line[2 * static_cast<size_t>(r)];
      profile[static_cast<size_t>(nr + r)] = dline[2 * static_cast<size_t>(r)];
    }
    std::vector<double2> seeds(segs.size() * static_cast<size_t>(max_ell),
                               make_double2(0.0, 0.0));
    for (size_t k = 0; k < segs.size(); ++k) {
      const SegmentDesc& sd = h_seg[static_cast<size_t>(segs[k])];
      for (size_t i = 0; i < ell.size(); ++i) {
        if (m[i] != sd.m) continue;
        double2& v = seeds[k * static_cast<size_t>(max_ell) +
                           static_cast<size_t>(ell[i] - sd.ell_min)];
        v.x += re[i];
        v.y += im[i];
      }
    }
    DeviceArray<double2> d_seeds;
    DeviceArray<double> d_profile;
    DeviceArray<unsigned long long> d_worst;
    alloc(d_seeds, seeds.size());
    alloc(d_profile, profile.size());
    alloc(d_worst, 1);
    check(cudaMemcpyAsync(d_seeds.ptr, seeds.data(), seeds.size() * sizeof(double2),
                          cudaMemcpyHostToDevice, stream),
          "upload seeds");
    check(cudaMemcpyAsync(d_profile.ptr, profile.data(),
                          profile.size() * sizeof(double), cudaMemcpyHostToDevice,
                          stream),
          "upload profile");
    check(cudaMemsetAsync(d_worst.ptr, 0, sizeof(unsigned long long), stream),
          "zero residual");
    check(cudaMemsetAsync(d_flag.ptr, 0, sizeof(int), stream), "zero flag");
    GaussianLaunch g{};
    g.y = y.ptr;
    g.segments = d_seg.ptr + segs.front();
    g.segment_count = static_cast<int>(segs.size());
    g.instance = h_inst[static_cast<size_t>(instance)];
    g.matrices = d_mat.ptr;
    g.trig = d_trig.ptr;
    g.seeds = d_seeds.ptr;
    g.profile = d_profile.ptr;
    g.max_ell = max_ell;
    g.worst_residual = d_worst.ptr;
    g.singular = d_flag.ptr;
    check(launch_gaussian_band(g, stream), "Gaussian initial data");
    unsigned long long bits = 0;
    int singular = 0;
    check(cudaMemcpyAsync(&bits, d_worst.ptr, sizeof(bits), cudaMemcpyDeviceToHost,
                          stream),
          "read residual");
    check(cudaMemcpyAsync(&singular, d_flag.ptr, sizeof(int), cudaMemcpyDeviceToHost,
                          stream),
          "read flag");
    check(cudaStreamSynchronize(stream), "Gaussian initial data");
    if (singular != 0) {
      throw std::runtime_error("singular Galerkin initialization matrix");
    }
    double worst = 0.0;
    std::memcpy(&worst, &bits, sizeof(worst));
    if (!std::isfinite(worst) || worst > 2.0e-12) {
      throw std::runtime_error(
          "Galerkin initial-time-derivative solve failed its residual check");
    }
    frozen_dev[static_cast<size_t>(instance)].release();
  }

  // RK4 steps whose three slope buffers (k1 / stage-4 input, k2, weighted
  // sum) are slopes[0, stride), [stride, 2 stride), [2 stride, 3 stride)
  // instead of kA / kB / acc.  Launches only: no allocation, no graph.
  void step_with_slopes(const std::vector<double>& dt, const int steps,
                        double2* slopes, const size_t stride) {
    if (steps < 0) throw std::invalid_argument("step count must be nonnegative");
    if (total_complex > stride) {
      throw std::invalid_argument("slope buffers are smaller than the band state");
    }
    set_dt(dt);
    for (int s = 0; s < steps; ++s) {
      for (const int kind : {kStage1, kStage2, kStage3, kStage4}) {
        for (StageLaunch g : groups) {
          g.stage = kind;
          g.kA = slopes;
          g.kB = slopes + stride;
          g.acc = slopes + 2 * stride;
          check(launch_stage(g, stream), "stage kernel");
        }
      }
    }
    check(cudaGetLastError(), "step");
  }

  void endpoint_modal(double* out, const size_t capacity, size_t* count,
                      const int memory) {
    const size_t n = h_seg.size() * 2 * static_cast<size_t>(max_ell);
    if (count != nullptr) *count = n;
    if (out == nullptr) return;
    if (capacity < n) {
      throw std::invalid_argument("endpoint buffer capacity is too small");
    }
    check(launch_endpoint_gather(y.ptr, d_seg.ptr, d_inst.ptr,
                                 static_cast<int>(h_seg.size()), max_ell,
                                 d_endpoint.ptr, stream),
          "endpoint gather");
    check(cudaMemcpyAsync(out, d_endpoint.ptr, n * sizeof(double2),
                          memory == TEUK_B200_HOST ? cudaMemcpyDeviceToHost
                                                   : cudaMemcpyDeviceToDevice,
                          stream),
          "endpoint copy");
    if (memory == TEUK_B200_HOST) {
      check(cudaStreamSynchronize(stream), "endpoint sync");
      check_kernel_error();
    }
  }

  void sample_endpoint(const int instance, teuk_b200_waveform_record* out,
                       const size_t capacity, size_t* count) {
    check_instance(instance);
    const InstancePlan& plan = plans[static_cast<size_t>(instance)];
    const Config& c = plan.config;
    const int ne_max = max_ell;
    std::vector<double2> gathered(h_seg.size() * 2 * static_cast<size_t>(ne_max));
    size_t n = 0;
    endpoint_modal(reinterpret_cast<double*>(gathered.data()), gathered.size(),
                   &n, TEUK_B200_HOST);
    std::vector<teuk_b200_waveform_record> records;
    const double scale[2] = {c.length * c.length, plan.horizon};
    // first-order field: modal coefficients straight from the band storage
    for (int boundary = 0; boundary < 2; ++boundary) {
      for (const ModePlan& mp : plan.modes) {
        if (!mp.parent) continue;
        const size_t base =
            (static_cast<size_t>(mp.segment) * 2 + static_cast<size_t>(boundary)) *
            static_cast<size_t>(ne_max);
        for (int l = 0; l < mp.n_ell; ++l) {
          const double2 v = gathered[base + static_cast<size_t>(l)];
          records.push_back({boundary, 1, mp.m, mp.ell_min + l, v.x, v.y,
                             scale[boundary] * v.x, scale[boundary] * v.y});
        }
      }
    }
    // second-order field: frozen in the linear pipeline; analyze the stored
    // endpoint values with the target band's transform.
    const int nt = c.ntheta;
    const auto& frozen = frozen_dev[static_cast<size_t>(instance)];
    std::vector<double2> slice(static_cast<size_t>(nt));
    for (int boundary = 0; boundary < 2; ++boundary) {
      const int r = boundary == 0 ? 0 : c.nr - 1;
      for (const ModePlan& mp : plan.modes) {
        if (!std::binary_search(c.targets.begin(), c.targets.end(), mp.m)) {
          continue;
        }
        std::fill(slice.begin(), slice.end(), make_double2(0.0, 0.0));
        if (frozen.ptr != nullptr) {
          const size_t offset =
              ((static_cast<size_t>(mp.mode_index) * kFieldCount + 12) *
                   static_cast<size_t>(c.nr) +
               static_cast<size_t>(r)) *
              static_cast<size_t>(nt);
          check(cudaMemcpy(slice.data(), frozen.ptr + offset,
                           static_cast<size_t>(nt) * sizeof(double2),
                           cudaMemcpyDeviceToHost),
                "second-order endpoint slice");
        }
        const int ell_min = std::max(2, std::abs(mp.m));
        const double pi = std::numbers::pi_v<double>;
        for (int ell = ell_min; ell <= c.ell_max_second; ++ell) {
          double re = 0.0, im = 0.0;
          for (int j = 0; j < nt; ++j) {
            const double a = 2.0 * pi * plan.weights[static_cast<size_t>(j)] *
                             spin_weighted_harmonic_theta(
                                 ell, mp.m, kSpinWeight,
                                 plan.theta[static_cast<size_t>(j)]);
            re += a * slice[static_cast<size_t>(j)].x;
            im += a * slice[static_cast<size_t>(j)].y;
          }
          records.push_back({boundary, 2, mp.m, ell, re, im,
                             scale[boundary] * re, scale[boundary] * im});
        }
      }
    }
    if (count != nullptr) *count = records.size();
    if (records.size() > capacity) {
      throw std::invalid_argument("waveform record capacity is too small");
    }
    std::copy(records.begin(), records.end(), out);
  }

  size_t device_bytes() const {
    return 4 * total_complex * sizeof(double2) + d_nodal.count * sizeof(double2) +
           h_mat.size() * sizeof(double) + h_trig.size() * sizeof(double) +
           h_tiles.size() * sizeof(TileDesc) + h_seg.size() * sizeof(SegmentDesc) +
           h_strips.size() * sizeof(TileDesc) + d_coef.count * sizeof(double) +
           d_nodes.count * sizeof(double) +
           d_endpoint.count * sizeof(double2);
  }
};

}  // namespace teuk_b200

using teuk_b200::Batch;
using teuk_b200::guarded;

struct teuk_b200_batch {
  std::unique_ptr<Batch> batch;
  // or: identical second-order solves with the Unrestricted source from
  // t = 0, the replicas of one nodal pipeline
  std::unique_ptr<teuk_b200::NodalPipeline> nodal;
  double time = 0.0;
};
struct teuk_b200_pipeline {
  // exactly one of the two is set: the band-storage batch of one solve for
  // the linear policy, the nodal pipeline for second-order source policies
  std::unique_ptr<Batch> batch;
  std::unique_ptr<teuk_b200::NodalPipeline> nodal;
};

namespace {

void require(const bool condition, const char* message) {
  if (!condition) throw std::invalid_argument(message);
}

void require_device() {
  int device_count = 0;
  const cudaError_t err = cudaGetDeviceCount(&device_count);
  if (err != cudaSuccess) {
    throw teuk_b200::DeviceError(std::string("cudaGetDeviceCount: ") +
                                 cudaGetErrorString(err));
  }
  if (device_count <= 0) {
    throw teuk_b200::DeviceError("no CUDA device is visible");
  }
}

// EndpointWaveformSampler::sample over a nodal state
// (include/teuk/waveform_output.hpp:75-160): psi at the two radial ends,
// analysed with the first-order band for parents and the second-order band
// for targets.
void sample_nodal_endpoint(teuk_b200::NodalPipeline& nodal,
                           teuk_b200_waveform_record* out,
                           const size_t capacity, size_t* count,
                           const int replica = 0) {
  using namespace teuk_b200;
  const InstancePlan& plan = nodal.plan();
  const Config& c = plan.config;
  const int nt = c.ntheta;
  const double pi = std::numbers::pi_v<double>;
  const double scale[2] = {c.length * c.length, plan.horizon};
  std::vector<teuk_b200_waveform_record> records;
  std::vector<double2> slice;
  for (int order = 1; order <= 2; ++order) {
    const int field = order == 1 ? 2 : 12;
    const std::vector<int>& members = order == 1 ? c.parents : c.targets;
    const int ell_max = order == 1 ? c.ell_max_first : c.ell_max_second;
    for (int boundary = 0; boundary < 2; ++boundary) {
      nodal.endpoint_slice(field, boundary == 0 ? 0 : c.nr - 1, slice, replica);
      for (size_t mode = 0; mode < c.modes.size(); ++mode) {
        const int m = c.modes[mode];
        if (!std::binary_search(members.begin(), members.end(), m)) continue;
        const int ell_min = std::max(2, std::abs(m));
        for (int ell = ell_min; ell <= ell_max; ++ell) {
          double re = 0.0, im = 0.0;
          for (int j = 0; j < nt; ++j) {
            const double a = 2.0 * pi * plan.weights[static_cast<size_t>(j)] *
                             spin_weighted_harmonic_theta(
                                 ell, m, kSpinWeight,
                                 plan.theta[static_cast<size_t>(j)]);
            const double2 v = slice[mode * static_cast<size_t>(nt) +
                                    static_cast<size_t>(j)];
            re += a * v.x;
            im += a * v.y;
          }
          records.push_back({boundary, order, m, ell, re, im,
                             scale[boundary] * re, scale[boundary] * im});
        }
      }
    }
  }
  if (count != nullptr) *count = records.size();
  if (records.size() > capacity) {
    throw std::invalid_argument("waveform record capacity is too small");
  }
  std::copy(records.begin(), records.end(), out);
}

void fill_shape(const teuk_b200::InstancePlan& plan, size_t shape[4]) {
  shape[0] = plan.config.modes.size();
  shape[1] = teuk_b200::kFieldCount;
  shape[2] = static_cast<size_t>(plan.config.nr);
  shape[3] = static_cast<size_t>(plan.config.ntheta);
}

void restore_activation(teuk_b200::InstancePlan& plan,
                        const teuk_b200_activation& s) {
  // SpatialPipeline::validate_source_activation_state
  // (include/teuk/spatial_pipeline.hpp:1225-1235)
  if (s.consecutive_passes < 0 || !std::isfinite(s.activation_time) ||
      !std::isfinite(s.last_eligibility_time) ||
      (s.active != 0 && s.activation_time < 0.0) ||
      (s.active == 0 && s.activation_time != -1.0) ||
      s.last_eligibility_time < -1.0) {
    throw std::invalid_argument("invalid second-order source activation state");
  }
  plan.active = s.active != 0 ? 1 : 0;
  plan.activation_time = s.activation_time;
  plan.consecutive_passes = s.consecutive_passes;
  plan.last_eligibility_time = s.last_eligibility_time;
}

void reset_activation(teuk_b200::InstancePlan& plan) {
  plan.active = 0;
  plan.activation_time = -1.0;
  plan.consecutive_passes = 0;
  plan.last_eligibility_time = -1.0;
  const auto& c = plan.config;
  if (c.source_mode == TEUK_B200_SOURCE_UNRESTRICTED &&
      c.source_start_time == 0.0) {
    plan.active = 1;
    plan.activation_time = 0.0;
    plan.consecutive_passes = c.required_passes;
  }
}

void initialize_gaussian(Batch& b, const int instance,
                         const teuk_b200_gaussian* pulse) {
  b.check_instance(instance);
  require(pulse != nullptr, "null Gaussian pulse");
  require(pulse->mode_count >= 0 &&
              (pulse->mode_count == 0 || pulse->modes != nullptr),
          "Gaussian mode list pointer/count mismatch");
  std::vector<int> ell, m;
  std::vector<double> re, im;
  for (int i = 0; i < pulse->mode_count; ++i) {
    ell.push_back(pulse->modes[i].ell);
    m.push_back(pulse->modes[i].m);
    re.push_back(pulse->modes[i].amplitude_real);
    im.push_back(pulse->modes[i].amplitude_imag);
  }
  b.gaussian_device(instance, pulse->center, pulse->width,
                    pulse->compact_support != 0, ell, m, re, im);
  reset_activation(b.plans[static_cast<size_t>(instance)]);
}

void initialize_nodal_gaussian(teuk_b200::NodalPipeline& p,
                               const teuk_b200_gaussian* pulse,
                               const int replica = -1) {
  require(pulse != nullptr, "null Gaussian pulse");
  require(pulse->mode_count >= 0 &&
              (pulse->mode_count == 0 || pulse->modes != nullptr),
          "Gaussian mode list pointer/count mismatch");
  std::vector<int> ell, m;
  std::vector<double> re, im;
  for (int i = 0; i < pulse->mode_count; ++i) {
    ell.push_back(pulse->modes[i].ell);
    m.push_back(pulse->modes[i].m);
    re.push_back(pulse->modes[i].amplitude_real);
    im.push_back(pulse->modes[i].amplitude_imag);
  }
  std::vector<double> nodal;
  teuk_b200::gaussian_initial_state(p.plan(), pulse->center, pulse->width,
                                    pulse->compact_support != 0, ell, m, re,
                                    im, nodal);
  if (replica >= 0) {  // one replica of a replicated pipeline
    p.set_replica_state(replica, nodal.data(), TEUK_B200_HOST);
    return;
  }
  p.set_state(nodal.data(), TEUK_B200_HOST);
  p.reset_activation();
}


// Device bytes one linear solve holds inside a batch: four band buffers
// (padded segments), its matrices, its row coefficients and the nodal
// import scratch.
size_t linear_footprint(const teuk_b200::InstancePlan& plan) {
  size_t complex_count = 0;
  size_t matrix = 0;
  for (const auto& mp : plan.modes) {
    if (!mp.parent) continue;
    const size_t count = static_cast<size_t>(plan.config.nr) * 3 *
                         static_cast<size_t>(mp.n_ell);
    complex_count += (count + 15) / 16 * 16;
    matrix += 2 * static_cast<size_t>(mp.n_ell * plan.config.ntheta);
  }
  // bands on the wide streaming kernel add a row of the wide node table
  bool wide = false;
  const int nt = plan.config.ntheta;
  for (const auto& mp : plan.modes) {
    if (!mp.parent) continue;
    const bool narrow =
        mp.n_ell <= teuk_b200::kStreamMaxEll && nt <= teuk_b200::kStreamMaxNodes;
    wide = wide || (!narrow && mp.n_ell <= teuk_b200::kWideMaxEll &&
                    nt <= teuk_b200::kWideMaxNodes && plan.config.reduction == 0);
  }
  const size_t node_record =
      teuk_b200::kNodeRecord + (wide ? teuk_b200::kWideMaxNodes : 0);
  return 4 * complex_count * sizeof(double2) + matrix * sizeof(double) +
         static_cast<size_t>(plan.config.nr) *
             (teuk_b200::kCoefRecord + node_record) * sizeof(double) +
         plan.value_count() * sizeof(double2);
}

double wall_seconds() {
  return std::chrono::duration<double>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct ServerRequest {
  uint64_t id = 0;
  teuk_b200::Config config;
  teuk_b200::InstancePlan plan;  // validated at submit, reused by rebuilds
  std::vector<teuk_b200_gaussian_mode> modes;
  teuk_b200_gaussian pulse{};
  double dt = 0.0;
  int steps = 0;
  int done = 0;
  int slot = -1;  // instance index in the current batch, -1 if not in it
  size_t footprint = 0;
  double points = 0.0;  // modes * nr * ntheta
  double submit_time = 0.0;
  double finish_time = -1.0;
  std::vector<teuk_b200_waveform_record> records;
  // Second-order (ConstraintAware / Unrestricted) requests: their own nodal
  // pipeline on its own stream, stepped beside the batch in every server
  // step; `time` advances by dt per step as in teuk_b200_step.
  bool second_order = false;
  double time = 0.0;
  std::unique_ptr<teuk_b200::NodalPipeline> nodal;
  cudaEvent_t joined = nullptr;  // end of this request's work of a step
  // or, when it shares a replicated pipeline: its group and replica slot
  struct NodalGroup* group = nullptr;
  int replica = -1;
  ~ServerRequest() {
    if (joined != nullptr) cudaEventDestroy(joined);
  }
};

// Second-order requests with the Unrestricted source from t = 0 that share
// their configuration, precision and dt are replicas of one nodal pipeline
// (stepped by the same launches; each replica's results equal the solve
// alone bit for bit).  The pipeline's room grows by doubling; a retiring
// member's slot takes the last replica's state.
struct NodalGroup {
  std::string key;
  teuk_b200::InstancePlan plan;
  double dt = 0.0;
  double time = 0.0;  // the source is on throughout: the RHS does not depend on it
  std::unique_ptr<teuk_b200::NodalPipeline> pipe;
  std::vector<ServerRequest*> members;  // replica k = members[k]
  cudaEvent_t joined = nullptr;
  ~NodalGroup() {
    pipe.reset();
    if (joined != nullptr) cudaEventDestroy(joined);
  }
};

// Text key of everything a replicated pipeline shares.
std::string nodal_group_key(const teuk_b200::Config& c, const int precision,
                            const double dt) {
  std::string k;
  const auto num = [&](const double v) {
    char buf[40];
    std::snprintf(buf, sizeof(buf), "%a,", v);
    k += buf;
  };
  const auto ints = [&](const std::vector<int>& v) {
    for (const int x : v) k += std::to_string(x) + " ";
    k += ";";
  };
  num(c.mass); num(c.spin); num(c.length); num(c.damping); num(c.dissipation);
  num(c.source_start_time); num(c.constraint_tolerance); num(dt);
  k += std::to_string(c.nr) + "," + std::to_string(c.ntheta) + "," +
       std::to_string(c.ell_max_first) + "," + std::to_string(c.ell_max_second) +
       "," + std::to_string(c.reduction) + "," + std::to_string(c.disc) + "," +
       std::to_string(c.source_mode) + "," + std::to_string(c.required_passes) +
       "," + std::to_string(precision) + ";";
  ints(c.modes); ints(c.parents); ints(c.targets);
  return k;
}

// Continuous batching over Batch: admitted solves share one batched RK4
// step; a change of membership rebuilds the batch layout and moves the band
// state of every continuing solve into it on the device.
class Server {
 public:
  explicit Server(const teuk_b200_server_options& o) : options_(o) {
    if (o.abi_version != TEUK_B200_ABI_VERSION) {
      throw std::invalid_argument("teuk_b200_server_options.abi_version mismatch");
    }
    if (o.hbm_budget_bytes == 0) {
      throw std::invalid_argument("server HBM budget must be positive");
    }
    if (o.max_active < 0) {
      throw std::invalid_argument("server max_active must be nonnegative");
    }
    if (o.precision != TEUK_B200_PRECISION_FP64 &&
        o.precision != TEUK_B200_PRECISION_SPLIT) {
      throw std::invalid_argument("unknown transform precision");
    }
    require_device();
    teuk_b200::check(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking),
                     "cudaStreamCreate");
    // The band arena's own memory pool: blocks it frees stay reserved for
    // the next layout (no release back to the driver until the server
    // ends).
    int device = 0;
    teuk_b200::check(cudaGetDevice(&device), "cudaGetDevice");
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    teuk_b200::check(cudaMemPoolCreate(&pool_, &props), "cudaMemPoolCreate");
    unsigned long long keep = ~0ull;
    teuk_b200::check(
        cudaMemPoolSetAttribute(pool_, cudaMemPoolAttrReleaseThreshold, &keep),
        "memory pool release threshold");
    arena_.pool = pool_;
    arena_.stream = stream_;
    arena_.cap = std::max<size_t>(
        1, o.hbm_budget_bytes / (4 * sizeof(double2)));
    // Warm the pool: map its first block now instead of inside the first
    // layout changes (a driver allocation can take tens to hundreds of ms).
    const size_t warm = std::min<size_t>(o.hbm_budget_bytes, size_t{4} << 30);
    void* block = nullptr;
    teuk_b200::check(cudaMallocFromPoolAsync(&block, warm, pool_, stream_),
                     "memory pool warm-up");
    teuk_b200::check(cudaFreeAsync(block, stream_), "memory pool warm-up");
    teuk_b200::check(cudaStreamSynchronize(stream_), "memory pool warm-up");
  }
  ~Server() {
    batch_.reset();
    arena_.release();  // stream-ordered frees into the pool
    if (stream_ != nullptr) cudaStreamSynchronize(stream_);
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
    if (stream_ != nullptr) cudaStreamDestroy(stream_);
    if (pool_ != nullptr) cudaMemPoolDestroy(pool_);
  }

  uint64_t submit(const teuk_b200_config& raw, const teuk_b200_gaussian& pulse,
                  const double dt, const int steps) {
    auto r = std::make_shared<ServerRequest>();
    r->config = teuk_b200::to_config(raw);
    r->plan = teuk_b200::build_instance_plan(r->config);
    const teuk_b200::InstancePlan& plan = r->plan;
    r->second_order = r->config.source_mode != TEUK_B200_SOURCE_DISABLED;
    if (!std::isfinite(dt) || !(dt > 0.0)) {
      throw std::invalid_argument("pipeline step requires finite positive time data");
    }
    if (steps < 0) throw std::invalid_argument("step count must be nonnegative");
    if (pulse.mode_count < 0 || (pulse.mode_count > 0 && pulse.modes == nullptr)) {
      throw std::invalid_argument("Gaussian mode list pointer/count mismatch");
    }
    r->footprint = r->second_order ? teuk_b200::nodal_footprint_bytes(plan)
                                   : linear_footprint(plan);
    if (r->footprint > options_.hbm_budget_bytes) {
      throw std::invalid_argument("solve footprint exceeds the server HBM budget");
    }
    r->modes.assign(pulse.modes, pulse.modes + pulse.mode_count);
    r->pulse = pulse;
    r->dt = dt;
    r->steps = steps;
    r->points = static_cast<double>(r->config.modes.size()) * r->config.nr *
                r->config.ntheta;
    r->id = next_id_++;
    r->submit_time = wall_seconds();
    requests_[r->id] = r;
    queue_.push_back(r);
    return r->id;
  }

  int advance(const int steps) {
    if (steps < 0) throw std::invalid_argument("step count must be nonnegative");
    retire();
    admit();
    pending_ = 0;
    for (int s = 0; s < steps && !active_.empty(); ++s) {
      step_once();
      retire();
      admit();
    }
    collect_step_times();
    return static_cast<int>(active_.size());
  }

  const ServerRequest& result(const uint64_t id) const {
    const auto it = requests_.find(id);
    if (it == requests_.end()) throw std::invalid_argument("unknown request id");
    if (it->second->finish_time < 0.0) {
      throw std::invalid_argument("request is not finished");
    }
    return *it->second;
  }

  teuk_b200_server_stats stats() const {
    teuk_b200_server_stats st{};
    st.queued = static_cast<int>(queue_.size());
    st.active = static_cast<int>(active_.size());
    st.finished = finished_;
    st.steps = steps_run_;
    st.grid_point_updates = grid_point_updates_;
    st.device_seconds = device_seconds_;
    st.resident_bytes = batch_ ? batch_->device_bytes() : 0;
    for (const auto& r : active_) {
      if (r->second_order) st.resident_bytes += r->footprint;
    }
    st.rebuilds = rebuilds_;
    st.rebuild_seconds = rebuild_seconds_;
    return st;
  }

 private:
  void admit() {
    bool changed = membership_changed_;
    while (!queue_.empty()) {
      const auto& r = queue_.front();
      if (options_.max_active > 0 &&
          static_cast<int>(active_.size()) >= options_.max_active) {
        break;
      }
      if (active_bytes_ + r->footprint > options_.hbm_budget_bytes) break;
      active_bytes_ += r->footprint;
      if (r->second_order && groupable(*r)) {
        join_group(*r);
      } else if (r->second_order) {
        start_nodal(*r);
      } else {
        changed = true;
      }
      active_.push_back(r);
      queue_.pop_front();
    }
    if (changed) rebuild();
    membership_changed_ = false;
  }

  // A second-order request gets its nodal pipeline, on its own stream, and
  // its Gaussian initial data when it is admitted.
  void start_nodal(ServerRequest& r) {
    r.nodal = std::make_unique<teuk_b200::NodalPipeline>(r.plan, options_.precision);
    teuk_b200_gaussian pulse = r.pulse;
    pulse.modes = r.modes.data();
    initialize_nodal_gaussian(*r.nodal, &pulse);
    teuk_b200::check(cudaEventCreateWithFlags(&r.joined, cudaEventDisableTiming),
                     "cudaEventCreate");
    r.time = 0.0;
  }

  static bool groupable(const ServerRequest& r) {
    return r.config.source_mode == TEUK_B200_SOURCE_UNRESTRICTED &&
           r.config.source_start_time == 0.0;
  }

  // Adds a second-order request to its group as the next replica, growing
  // the group's pipeline (state of the members moved on the device) when
  // it has no room left.
  void join_group(ServerRequest& r) {
    const std::string key = nodal_group_key(r.config, options_.precision, r.dt);
    NodalGroup* g = nullptr;
    for (const auto& grp : groups_) {
      if (grp->key == key) g = grp.get();
    }
    if (g == nullptr) {
      auto created = std::make_unique<NodalGroup>();
      created->key = key;
      created->plan = r.plan;
      created->dt = r.dt;
      teuk_b200::check(
          cudaEventCreateWithFlags(&created->joined, cudaEventDisableTiming),
          "cudaEventCreate");
      g = created.get();
      groups_.push_back(std::move(created));
    }
    const int k = static_cast<int>(g->members.size());
    if (!g->pipe || k + 1 > g->pipe->replicas()) {
      collect_step_times();
      const int room = std::max(k + 1, g->pipe ? 2 * g->pipe->replicas() : 2);
      auto next = std::make_unique<teuk_b200::NodalPipeline>(
          g->plan, options_.precision, room);
      next->reset_activation();  // the source is on from t = 0
      next->set_active_replicas(k + 1);
      for (int i = 0; i < k; ++i) next->copy_replica_from(*g->pipe, i, i);
      g->pipe = std::move(next);
    } else {
      g->pipe->set_active_replicas(k + 1);
    }
    teuk_b200_gaussian pulse = r.pulse;
    pulse.modes = r.modes.data();
    initialize_nodal_gaussian(*g->pipe, &pulse, k);
    g->members.push_back(&r);
    r.group = g;
    r.replica = k;
  }

  // Records of a finished group member; the last replica moves into its
  // slot.  An empty group releases its pipeline.
  void leave_group(ServerRequest& r, teuk_b200_waveform_record* out,
                   const size_t capacity, size_t* count) {
    NodalGroup* g = r.group;
    collect_step_times();
    sample_nodal_endpoint(*g->pipe, out, capacity, count, r.replica);
    const int last = static_cast<int>(g->members.size()) - 1;
    if (r.replica != last) {
      g->pipe->copy_replica_from(*g->pipe, last, r.replica);
      g->members[static_cast<size_t>(r.replica)] = g->members[static_cast<size_t>(last)];
      g->members[static_cast<size_t>(r.replica)]->replica = r.replica;
    }
    g->members.pop_back();
    if (g->members.empty()) {
      g->pipe.reset();
    } else {
      g->pipe->set_active_replicas(static_cast<int>(g->members.size()));
    }
    r.group = nullptr;
    r.replica = -1;
  }

  std::vector<std::shared_ptr<ServerRequest>> linear_active() const {
    std::vector<std::shared_ptr<ServerRequest>> out;
    for (const auto& r : active_) {
      if (!r->second_order) out.push_back(r);
    }
    return out;
  }

  // New batch layout for the admitted set; continuing solves keep their
  // band state (device-to-device), new ones get their Gaussian data.
  void rebuild() {
    const auto linear = linear_active();
    if (linear.empty()) {
      collect_step_times();
      batch_.reset();
      return;
    }
    collect_step_times();
    const double t0 = wall_seconds();
    std::vector<teuk_b200::InstancePlan> plans;
    for (const auto& r : linear) plans.push_back(r->plan);
    auto next = std::make_unique<Batch>();
    next->options.precision = options_.precision;
    next->build_planned(std::move(plans), &arena_);
    // the coefficient tables were computed on the batch's build stream:
    // finish them before the server's stream takes over
    teuk_b200::check(cudaStreamSynchronize(next->stream), "batch build");
    next->stream = stream_;
    for (size_t i = 0; i < linear.size(); ++i) {
      ServerRequest& r = *linear[i];
      const int slot = static_cast<int>(i);
      if (r.slot >= 0 && batch_) {
        const auto& from = batch_->instance_segments[static_cast<size_t>(r.slot)];
        const auto& to = next->instance_segments[i];
        for (size_t k = 0; k < from.size(); ++k) {
          const auto& a = batch_->h_seg[static_cast<size_t>(from[k])];
          const auto& b = next->h_seg[static_cast<size_t>(to[k])];
          const size_t n = static_cast<size_t>(r.config.nr) * 3 *
                           static_cast<size_t>(a.n_ell);
          teuk_b200::check(
              cudaMemcpyAsync(next->y.ptr + b.offset, batch_->y.ptr + a.offset,
                              n * sizeof(double2), cudaMemcpyDeviceToDevice,
                              stream_),
              "move band state");
        }
        next->frozen_dev[i] =
            std::move(batch_->frozen_dev[static_cast<size_t>(r.slot)]);
      } else {
        teuk_b200_gaussian pulse = r.pulse;
        pulse.modes = r.modes.data();
        initialize_gaussian(*next, slot, &pulse);
      }
      r.slot = slot;
    }
    teuk_b200::check(cudaStreamSynchronize(stream_), "server rebuild");
    batch_ = std::move(next);
    arena_.current = 1 - arena_.current;
    ++rebuilds_;
    rebuild_seconds_ += wall_seconds() - t0;
  }

  // One batched step, bracketed by a pair of events; the host does not
  // wait for it (a retirement's endpoint read is the next synchronisation).
  //
  // Second-order requests step on their own streams between the same pair
  // of events: they wait for the step's start event and the server stream
  // waits for each of them before the stop event, so the device time of a
  // step covers the batch and every nodal pipeline running beside it.
  void step_once() {
    std::vector<double> dts;
    for (const auto& r : active_) {
      if (!r->second_order) dts.push_back(r->dt);
    }
    while (events_.size() < 2 * static_cast<size_t>(pending_ + 1)) {
      cudaEvent_t e = nullptr;
      teuk_b200::check(cudaEventCreate(&e), "cudaEventCreate");
      events_.push_back(e);
    }
    cudaEvent_t start = events_[2 * pending_];
    teuk_b200::check(cudaEventRecord(start, stream_), "event");
    if (batch_ && !dts.empty()) batch_->step(dts, 1, options_.graph != 0);
    for (const auto& r : active_) {
      if (!r->second_order || r->group != nullptr) continue;
      teuk_b200::check(cudaStreamWaitEvent(r->nodal->stream(), start, 0),
                       "nodal fork");
      r->nodal->step(r->time, r->dt);
      r->time += r->dt;
      teuk_b200::check(cudaEventRecord(r->joined, r->nodal->stream()), "event");
      teuk_b200::check(cudaStreamWaitEvent(stream_, r->joined, 0), "nodal join");
    }
    for (const auto& g : groups_) {
      if (g->members.empty()) continue;
      teuk_b200::check(cudaStreamWaitEvent(g->pipe->stream(), start, 0),
                       "group fork");
      g->pipe->step(g->time, g->dt);
      g->time += g->dt;
      teuk_b200::check(cudaEventRecord(g->joined, g->pipe->stream()), "event");
      teuk_b200::check(cudaStreamWaitEvent(stream_, g->joined, 0), "group join");
    }
    teuk_b200::check(cudaEventRecord(events_[2 * pending_ + 1], stream_),
                     "event");
    ++pending_;
    ++steps_run_;
    for (const auto& r : active_) {
      ++r->done;
      grid_point_updates_ += r->points;
    }
  }

  void collect_step_times() {
    if (pending_ == 0) return;
    teuk_b200::check(cudaStreamSynchronize(stream_), "server steps");
    if (batch_) batch_->check_kernel_error();
    for (int i = 0; i < pending_; ++i) {
      float ms = 0.0f;
      teuk_b200::check(cudaEventElapsedTime(&ms, events_[2 * i],
                                            events_[2 * i + 1]),
                       "event time");
      device_seconds_ += 1e-3 * ms;
    }
    pending_ = 0;
  }

  void retire() {
    std::vector<std::shared_ptr<ServerRequest>> keep;
    for (const auto& r : active_) {
      if (r->done < r->steps) {
        keep.push_back(r);
        continue;
      }
      const teuk_b200::Config& c = r->config;
      size_t count = 0;
      r->records.resize(2 * c.modes.size() *
                        static_cast<size_t>(c.ell_max_first + c.ell_max_second + 2));
      if (r->group != nullptr) {
        leave_group(*r, r->records.data(), r->records.size(), &count);
      } else if (r->second_order) {
        collect_step_times();
        sample_nodal_endpoint(*r->nodal, r->records.data(), r->records.size(),
                              &count);
        r->nodal.reset();
      } else {
        batch_->sample_endpoint(r->slot, r->records.data(), r->records.size(),
                                &count);
        membership_changed_ = true;
      }
      r->records.resize(count);
      r->finish_time = wall_seconds();
      r->slot = -1;
      active_bytes_ -= r->footprint;
      ++finished_;
    }
    active_.swap(keep);
  }

  teuk_b200_server_options options_;
  cudaStream_t stream_ = nullptr;
  std::vector<cudaEvent_t> events_;  // start / stop pairs of pending steps
  teuk_b200::StateArena arena_;      // band buffers reused across layouts
  cudaMemPool_t pool_ = nullptr;     // the arena's memory pool
  int pending_ = 0;
  std::unique_ptr<Batch> batch_;
  std::vector<std::unique_ptr<NodalGroup>> groups_;  // replicated second order
  std::deque<std::shared_ptr<ServerRequest>> queue_;
  std::vector<std::shared_ptr<ServerRequest>> active_;
  std::unordered_map<uint64_t, std::shared_ptr<ServerRequest>> requests_;
  uint64_t next_id_ = 1;
  size_t active_bytes_ = 0;
  bool membership_changed_ = false;
  int finished_ = 0;
  int rebuilds_ = 0;
  double rebuild_seconds_ = 0.0;
  long long steps_run_ = 0;
  double grid_point_updates_ = 0.0;
  double device_seconds_ = 0.0;
};

}  // namespace

extern "C" {

const char* teuk_b200_last_error(void) {
  return teuk_b200::g_last_error.c_str();
}

int teuk_b200_abi_version(void) { return TEUK_B200_ABI_VERSION; }

int teuk_b200_set_device(int device) {
  return guarded([&] {
    int count = 0;
    teuk_b200::check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
    require(device >= 0 && device < count, "CUDA device index out of range");
    teuk_b200::check(cudaSetDevice(device), "cudaSetDevice");
  });
}

int teuk_b200_get_device(int* device) {
  return guarded([&] {
    require(device != nullptr, "null argument");
    teuk_b200::check(cudaGetDevice(device), "cudaGetDevice");
  });
}

namespace {
teuk_b200_batch_options checked_options(const teuk_b200_batch_options* o) {
  teuk_b200_batch_options out{TEUK_B200_ABI_VERSION, TEUK_B200_KERNEL_AUTO,
                              TEUK_B200_PRECISION_FP64, 0, 0};
  if (o == nullptr) return out;
  if (o->abi_version != TEUK_B200_ABI_VERSION) {
    throw std::invalid_argument("teuk_b200_batch_options.abi_version mismatch");
  }
  if (o->stage_kernel != TEUK_B200_KERNEL_AUTO &&
      o->stage_kernel != TEUK_B200_KERNEL_TILE) {
    throw std::invalid_argument("unknown stage kernel choice");
  }
  if (o->precision != TEUK_B200_PRECISION_FP64 &&
      o->precision != TEUK_B200_PRECISION_SPLIT) {
    throw std::invalid_argument("unknown transform precision");
  }
  if (o->strip_rows != 0 && o->strip_rows < teuk_b200::kStripMinRows) {
    throw std::invalid_argument("strip_rows must be 0 or at least 64");
  }
  if (o->autotune != 0 && o->autotune != 1) {
    throw std::invalid_argument("autotune must be 0 or 1");
  }
  return *o;
}

int create_pipeline(const teuk_b200_config* config,
                    const teuk_b200_batch_options* options,
                    teuk_b200_pipeline** out) {
  return guarded([&] {
    require(config != nullptr && out != nullptr, "null argument");
    const teuk_b200_batch_options opts = checked_options(options);
    auto p = std::make_unique<teuk_b200_pipeline>();
    const teuk_b200::Config c = teuk_b200::to_config(*config);
    if (c.source_mode != TEUK_B200_SOURCE_DISABLED) {
      const teuk_b200::InstancePlan plan = teuk_b200::build_instance_plan(c);
      require_device();
      p->nodal = std::make_unique<teuk_b200::NodalPipeline>(plan, opts.precision);
    } else {
      p->batch = std::make_unique<Batch>();
      p->batch->options = opts;
      p->batch->build({c});
    }
    *out = p.release();
  });
}
}  // namespace

int teuk_b200_create(const teuk_b200_config* config,
                     teuk_b200_pipeline** out) {
  return create_pipeline(config, nullptr, out);
}

int teuk_b200_create_with_options(const teuk_b200_config* config,
                                  const teuk_b200_batch_options* options,
                                  teuk_b200_pipeline** out) {
  return create_pipeline(config, options, out);
}

int teuk_b200_test_withhold_chunk(int chunk) {
  return guarded([&] {
    require(chunk >= -1, "chunk must be -1 (off) or a chunk index");
    teuk_b200::g_test_withhold_chunk.store(chunk);
  });
}

int teuk_b200_destroy(teuk_b200_pipeline* pipeline) {
  delete pipeline;
  return TEUK_B200_OK;
}

int teuk_b200_shape(const teuk_b200_pipeline* p, size_t shape[4]) {
  return guarded([&] {
    require(p != nullptr && shape != nullptr, "null argument");
    fill_shape(p->nodal ? p->nodal->plan() : p->batch->plans[0], shape);
  });
}

int teuk_b200_set_state(teuk_b200_pipeline* p, const double* state,
                        size_t count, int memory) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (p->nodal) {
      require(count == p->nodal->value_count(),
              "state complex count does not match shape");
      require(state != nullptr, "null state pointer");
      p->nodal->set_state(state, memory);
      return;
    }
    p->batch->set_state(0, state, count, memory);
  });
}

int teuk_b200_get_state(teuk_b200_pipeline* p, double* state, size_t count,
                        int memory) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (p->nodal) {
      require(count == p->nodal->value_count(),
              "state complex count does not match shape");
      require(state != nullptr, "null state pointer");
      p->nodal->get_state(state, memory);
      return;
    }
    p->batch->get_state(0, state, count, memory);
  });
}

int teuk_b200_evaluate_rhs(teuk_b200_pipeline* p, const double* stage,
                           double* output, size_t count, double time,
                           int memory) {
  return guarded([&] {
    require(p != nullptr && stage != nullptr && output != nullptr,
            "null argument");
    require(std::isfinite(time), "stage time must be finite");
    if (p->nodal) {
      require(count == p->nodal->value_count(),
              "state complex count does not match shape");
      p->nodal->evaluate_rhs(stage, output, memory, time);
      return;
    }
    p->batch->evaluate_rhs(0, stage, output, count, memory);
  });
}

int teuk_b200_step(teuk_b200_pipeline* p, double time, double dt, int steps) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (!std::isfinite(time) || !std::isfinite(dt) || time < 0.0 ||
        !(dt > 0.0)) {
      throw std::invalid_argument(
          "pipeline step requires finite positive time data");
    }
    if (p->nodal) {
      require(steps >= 0, "step count must be nonnegative");
      // the driver loop of the reference: time advances by dt per step
      double t = time;
      for (int s = 0; s < steps; ++s) {
        p->nodal->step(t, dt);
        t += dt;
      }
      teuk_b200::check(cudaStreamSynchronize(p->nodal->stream()), "step");
      return;
    }
    p->batch->step({dt}, steps, false);
    teuk_b200::check(cudaStreamSynchronize(p->batch->stream), "step");
    p->batch->check_kernel_error();
  });
}

int teuk_b200_step_static_scratch(teuk_b200_pipeline* p, double time,
                                  double dt, int steps) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (p->nodal) {
      throw teuk_b200::Unsupported(
          "static-scratch steps cover the linear (disabled-source) pipeline "
          "only");
    }
    if (!std::isfinite(time) || !std::isfinite(dt) || time < 0.0 ||
        !(dt > 0.0)) {
      throw std::invalid_argument(
          "pipeline step requires finite positive time data");
    }
    Batch& b = *p->batch;
    if (b.total_complex > teuk_b200::kStaticSlopeCapacity) {
      throw std::invalid_argument(
          "band state of " + std::to_string(b.total_complex) +
          " complex values exceeds the static scratch capacity of " +
          std::to_string(teuk_b200::kStaticSlopeCapacity) +
          " per slope buffer; use teuk_b200_step");
    }
    double2* slopes = nullptr;
    teuk_b200::check(teuk_b200::static_slope_buffers(&slopes),
                     "static scratch address");
    b.step_with_slopes({dt}, steps, slopes, teuk_b200::kStaticSlopeCapacity);
    teuk_b200::check(cudaStreamSynchronize(b.stream), "step");
    b.check_kernel_error();
  });
}

int teuk_b200_initialize_gaussian(teuk_b200_pipeline* p,
                                  const teuk_b200_gaussian* pulse) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (p->nodal) {
      initialize_nodal_gaussian(*p->nodal, pulse);
      return;
    }
    initialize_gaussian(*p->batch, 0, pulse);
  });
}

int teuk_b200_sample_endpoint(teuk_b200_pipeline* p,
                              teuk_b200_waveform_record* out,
                              size_t capacity, size_t* count) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (p->nodal) {
      sample_nodal_endpoint(*p->nodal, out, capacity, count);
      return;
    }
    p->batch->sample_endpoint(0, out, capacity, count);
  });
}

int teuk_b200_get_activation(const teuk_b200_pipeline* p,
                             teuk_b200_activation* out) {
  return guarded([&] {
    require(p != nullptr && out != nullptr, "null argument");
    if (p->nodal) {
      const auto s = p->nodal->activation();
      out->active = s.active ? 1 : 0;
      out->activation_time = s.activation_time;
      out->consecutive_passes = s.consecutive_passes;
      out->last_eligibility_time = s.last_eligibility_time;
      return;
    }
    const auto& plan = p->batch->plans[0];
    out->active = plan.active;
    out->activation_time = plan.activation_time;
    out->consecutive_passes = plan.consecutive_passes;
    out->last_eligibility_time = plan.last_eligibility_time;
  });
}

int teuk_b200_restore_activation(teuk_b200_pipeline* p,
                                 const teuk_b200_activation* state) {
  return guarded([&] {
    require(p != nullptr && state != nullptr, "null argument");
    if (p->nodal) {
      teuk_b200::InstancePlan scratch = p->nodal->plan();
      restore_activation(scratch, *state);  // validates like the reference
      p->nodal->restore_activation({scratch.active != 0,
                                    scratch.activation_time,
                                    scratch.consecutive_passes,
                                    scratch.last_eligibility_time});
      return;
    }
    restore_activation(p->batch->plans[0], *state);
  });
}

int teuk_b200_reset_activation(teuk_b200_pipeline* p) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (p->nodal) {
      p->nodal->reset_activation();
      return;
    }
    reset_activation(p->batch->plans[0]);
  });
}

int teuk_b200_set_stream(teuk_b200_pipeline* p, void* cuda_stream) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    if (p->nodal) {
      p->nodal->set_stream(static_cast<cudaStream_t>(cuda_stream));
      return;
    }
    p->batch->stream = cuda_stream != nullptr
                           ? static_cast<cudaStream_t>(cuda_stream)
                           : p->batch->own_stream;
  });
}

int teuk_b200_synchronize(teuk_b200_pipeline* p) {
  return guarded([&] {
    require(p != nullptr, "null pipeline");
    teuk_b200::check(cudaStreamSynchronize(p->nodal ? p->nodal->stream()
                                                     : p->batch->stream),
                     "synchronize");
    if (!p->nodal) p->batch->check_kernel_error();
  });
}

int teuk_b200_checkpoint_write(teuk_b200_pipeline* p, const char* directory,
                               double time_step, double time, uint64_t step) {
  return guarded([&] {
    require(p != nullptr && directory != nullptr, "null argument");
    const teuk_b200::InstancePlan& plan =
        p->nodal ? p->nodal->plan() : p->batch->plans[0];
    std::vector<double> state(2 * plan.value_count());
    teuk_b200::CheckpointActivation a;
    if (p->nodal) {
      p->nodal->get_state(state.data(), TEUK_B200_HOST);
      const auto s = p->nodal->activation();
      a = {s.active, s.activation_time, s.consecutive_passes,
           s.last_eligibility_time};
    } else {
      p->batch->get_state(0, state.data(), plan.value_count(), TEUK_B200_HOST);
      a = {plan.active != 0, plan.activation_time, plan.consecutive_passes,
           plan.last_eligibility_time};
    }
    teuk_b200::write_checkpoint(directory, plan, a, time_step, time, step,
                                state);
  });
}

int teuk_b200_checkpoint_load(teuk_b200_pipeline* p, const char* directory,
                              double time_step, double* time, uint64_t* step) {
  return guarded([&] {
    require(p != nullptr && directory != nullptr, "null argument");
    const teuk_b200::InstancePlan& plan =
        p->nodal ? p->nodal->plan() : p->batch->plans[0];
    const teuk_b200::CheckpointContents c =
        teuk_b200::read_checkpoint(directory, plan, time_step);
    const teuk_b200_activation a{c.activation.active ? 1 : 0,
                                 c.activation.activation_time,
                                 c.activation.consecutive_passes,
                                 c.activation.last_eligibility_time};
    if (p->nodal) {
      p->nodal->set_state(c.state.data(), TEUK_B200_HOST);
      p->nodal->restore_activation({a.active != 0, a.activation_time,
                                    a.consecutive_passes,
                                    a.last_eligibility_time});
    } else {
      p->batch->set_state(0, c.state.data(), plan.value_count(),
                          TEUK_B200_HOST);
      restore_activation(p->batch->plans[0], a);
    }
    if (time != nullptr) *time = c.time;
    if (step != nullptr) *step = c.step;
  });
}

namespace {

std::vector<std::string> override_list(const char* const* overrides,
                                       const int count) {
  require(count >= 0 && (count == 0 || overrides != nullptr),
          "override list pointer/count mismatch");
  std::vector<std::string> out;
  for (int i = 0; i < count; ++i) {
    require(overrides[i] != nullptr, "null override");
    out.emplace_back(overrides[i]);
  }
  return out;
}

void copy_path(char* dst, const std::string& src) {
  if (src.size() >= TEUK_B200_PATH_CAPACITY) {
    throw std::invalid_argument("configuration path exceeds the C ABI capacity");
  }
  std::memcpy(dst, src.c_str(), src.size() + 1);
}

}  // namespace

int teuk_b200_parse_run_config(const char* text, const char* const* overrides,
                               int override_count, teuk_b200_run_config* out) {
  return guarded([&] {
    require(text != nullptr && out != nullptr, "null argument");
    const teuk_b200::RunParameters run = teuk_b200::parse_run_configuration(
        text, override_list(overrides, override_count));
    const teuk_b200::Config c = teuk_b200::pipeline_config(run);
    // seeds only describe Gaussian initial data
    const auto seeds = run.initial_type == 0
                           ? teuk_b200::expanded_seeds(run)
                           : std::vector<teuk_b200::RunSeed>{};
    if (c.modes.size() > TEUK_B200_MAX_MODES ||
        seeds.size() > TEUK_B200_MAX_SEEDS) {
      throw std::invalid_argument("configuration exceeds the C ABI capacity");
    }
    teuk_b200_run_config r{};
    r.abi_version = TEUK_B200_ABI_VERSION;
    r.mass = c.mass;
    r.spin = c.spin;
    r.compactification_length = c.length;
    r.radial_points = c.nr;
    r.theta_nodes = c.ntheta;
    r.ell_max_first = c.ell_max_first;
    r.ell_max_second = c.ell_max_second;
    r.mode_count = static_cast<int>(c.modes.size());
    std::copy(c.modes.begin(), c.modes.end(), r.modes);
    r.parent_count = static_cast<int>(c.parents.size());
    std::copy(c.parents.begin(), c.parents.end(), r.parents);
    r.target_count = static_cast<int>(c.targets.size());
    std::copy(c.targets.begin(), c.targets.end(), r.targets);
    r.reduction_damping = c.damping;
    r.dissipation = c.dissipation;
    r.reduction = c.reduction;
    r.discretization = c.disc;
    r.source_mode = c.source_mode;
    r.source_start_time = c.source_start_time;
    r.normalized_constraint_tolerance = c.constraint_tolerance;
    r.required_consecutive_passes = c.required_passes;
    r.final_time = run.final_time;
    r.steps = run.steps;
    r.cfl = run.cfl;
    r.time_step = teuk_b200::run_time_step(run);
    r.initial_data_type = run.initial_type;
    const double horizon =
        c.length * c.length / teuk_b200::outer_horizon_radius(c.mass, c.spin);
    r.center = run.center_fraction * horizon;
    r.width = run.width_fraction * horizon;
    r.compact_support = run.compact_support ? 1 : 0;
    r.seed_count = static_cast<int>(seeds.size());
    for (size_t i = 0; i < seeds.size(); ++i) {
      r.seeds[i] = {seeds[i].ell, seeds[i].m, seeds[i].amplitude.real(),
                    seeds[i].amplitude.imag()};
    }
    copy_path(r.checkpoint_directory, run.checkpoint_directory);
    copy_path(r.output_directory, run.output_directory);
    r.diagnostic_every = run.diagnostic_every;
    r.checkpoint_every = run.checkpoint_every;
    *out = r;
  });
}

int teuk_b200_run_pipeline_config(const teuk_b200_run_config* run,
                                  teuk_b200_config* out) {
  return guarded([&] {
    require(run != nullptr && out != nullptr, "null argument");
    teuk_b200_config c{};
    c.abi_version = TEUK_B200_ABI_VERSION;
    c.mass = run->mass;
    c.spin = run->spin;
    c.compactification_length = run->compactification_length;
    c.radial_points = run->radial_points;
    c.theta_nodes = run->theta_nodes;
    c.ell_max_first = run->ell_max_first;
    c.ell_max_second = run->ell_max_second;
    c.mode_count = run->mode_count;
    c.modes = run->modes;
    c.parent_count = run->parent_count;
    c.parents = run->parents;
    c.target_count = run->target_count;
    c.targets = run->targets;
    c.reduction_damping = run->reduction_damping;
    c.dissipation = run->dissipation;
    c.reduction = run->reduction;
    c.discretization = run->discretization;
    c.source_mode = run->source_mode;
    c.source_start_time = run->source_start_time;
    c.normalized_constraint_tolerance = run->normalized_constraint_tolerance;
    c.required_consecutive_passes = run->required_consecutive_passes;
    *out = c;
  });
}

int teuk_b200_resolved_config(const char* text, const char* const* overrides,
                              int override_count, char* out, size_t capacity,
                              size_t* length) {
  return guarded([&] {
    require(text != nullptr, "null argument");
    const std::string resolved = teuk_b200::resolved_configuration_text(
        teuk_b200::parse_run_configuration(
            text, override_list(overrides, override_count)));
    if (length != nullptr) *length = resolved.size();
    if (out == nullptr) return;
    require(capacity > resolved.size(), "resolved configuration capacity is too small");
    std::memcpy(out, resolved.c_str(), resolved.size() + 1);
  });
}

int teuk_b200_diagnostics_sample(teuk_b200_pipeline* p,
                                 teuk_b200_diagnostics* out) {
  return guarded([&] {
    require(p != nullptr && out != nullptr, "null argument");
    using teuk_b200::DeviceArray;
    const teuk_b200::InstancePlan& plan =
        p->nodal ? p->nodal->plan() : p->batch->plans[0];
    const teuk_b200::Config& c = plan.config;
    cudaStream_t stream = p->nodal ? p->nodal->stream() : p->batch->stream;
    teuk_b200::DiagnosticsLaunch d{};
    if (p->nodal) {
      d.state = p->nodal->state_device();
      d.rhs = p->nodal->storage_rhs_device();
      d.source = p->nodal->source_device();
      d.forcing = p->nodal->forcing_device();
    } else {
      // nodal view of the band state; the linear pipeline never writes its
      // storage RHS, source or forcing, which therefore read as zero
      p->batch->assemble_nodal(0, p->batch->y.ptr, false);
      d.state = p->batch->nodal_scratch();
    }
    teuk_b200::check(teuk_b200::upload_nodal_sbp_constants(),
                     "upload SBP constants");
    DeviceArray<double> sums;
    DeviceArray<unsigned long long> maxima;
    DeviceArray<int> finite;
    sums.allocate(30);
    maxima.allocate(30);
    finite.allocate(8);
    const int ones[8] = {1, 1, 1, 1, 1, 1, 1, 1};
    teuk_b200::check(cudaMemsetAsync(sums.ptr, 0, 30 * sizeof(double), stream),
                     "zero sums");
    teuk_b200::check(
        cudaMemsetAsync(maxima.ptr, 0, 30 * sizeof(unsigned long long), stream),
        "zero maxima");
    teuk_b200::check(cudaMemcpyAsync(finite.ptr, ones, sizeof(ones),
                                     cudaMemcpyHostToDevice, stream),
                     "finite flags");
    d.modes = static_cast<int>(c.modes.size());
    d.nr = c.nr;
    d.nt = c.ntheta;
    d.disc = c.disc;
    d.inv_spacing = 1.0 / plan.spacing;
    d.sums = sums.ptr;
    d.maxima = maxima.ptr;
    d.finite = finite.ptr;
    teuk_b200::check(teuk_b200::launch_diagnostics(d, stream), "diagnostics");
    double h_sums[30];
    unsigned long long h_max[30];
    int h_finite[8];
    teuk_b200::check(cudaMemcpyAsync(h_sums, sums.ptr, sizeof(h_sums),
                                     cudaMemcpyDeviceToHost, stream),
                     "read sums");
    teuk_b200::check(cudaMemcpyAsync(h_max, maxima.ptr, sizeof(h_max),
                                     cudaMemcpyDeviceToHost, stream),
                     "read maxima");
    teuk_b200::check(cudaMemcpyAsync(h_finite, finite.ptr, sizeof(h_finite),
                                     cudaMemcpyDeviceToHost, stream),
                     "read flags");
    teuk_b200::check(cudaStreamSynchronize(stream), "diagnostics");
    teuk_b200_diagnostics r{};
    const size_t points = c.modes.size() * static_cast<size_t>(c.nr) *
                          static_cast<size_t>(c.ntheta);
    const double inv = 1.0 / static_cast<double>(points);
    const auto norm = [&](const int slot) {
      double m = 0.0;
      std::memcpy(&m, &h_max[slot], sizeof(m));
      return teuk_b200_norm{std::sqrt(h_sums[slot] * inv), std::sqrt(m)};
    };
    for (int f = 0; f < teuk_b200::kFieldCount; ++f) {
      r.state[f] = norm(f);
      r.rhs[f] = norm(teuk_b200::kFieldCount + f);
    }
    r.first_reduction_constraint = norm(26);
    r.second_reduction_constraint = norm(27);
    r.source_over_r3 = norm(28);
    r.forcing = norm(29);
    r.point_count = points;
    r.scri_finite = h_finite[6];
    r.horizon_finite = h_finite[7];
    r.all_finite = 1;
    for (const int f : h_finite) r.all_finite &= f != 0 ? 1 : 0;
    if (r.all_finite == 0) {
      // PipelineDiagnostics::nonfinite_message
      std::string message = "pipeline diagnostics found nonfinite values in";
      const char* names[8] = {" state", " rhs", " first-constraint",
                              " second-constraint", " source", " forcing",
                              " scri-endpoint", " horizon-endpoint"};
      for (int f = 0; f < 8; ++f) {
        if (h_finite[f] == 0) message += names[f];
      }
      throw std::runtime_error(message);
    }
    if (p->nodal) {
      const teuk_b200::ConstraintNorms& n = p->nodal->constraint_norms();
      for (int k = 0; k < 3; ++k) {
        r.constraint_absolute_maximum[k] = n.absolute_maximum[k];
        r.constraint_normalized_maximum[k] = n.normalized_maximum[k];
        r.constraint_weighted_rms[k] = n.weighted_rms[k];
        r.constraint_normalized_weighted[k] = n.normalized_weighted[k];
      }
      r.constraint_controlling_normalized = n.controlling_normalized;
      r.constraints_finite = n.all_finite ? 1 : 0;
      r.independent_reconstruction_constraint_maximum =
          p->nodal->independent_constraint_maximum();
      const auto a = p->nodal->activation();
      r.activation = {a.active ? 1 : 0, a.activation_time, a.consecutive_passes,
                      a.last_eligibility_time};
    } else {
      r.constraints_finite = 1;
      r.activation = {plan.active, plan.activation_time, plan.consecutive_passes,
                      plan.last_eligibility_time};
    }
    r.second_order_source_active = r.activation.active;
    *out = r;
  });
}

int teuk_b200_footprint_bytes(const teuk_b200_config* config, size_t* bytes) {
  return guarded([&] {
    require(config != nullptr && bytes != nullptr, "null argument");
    const auto plan =
        teuk_b200::build_instance_plan(teuk_b200::to_config(*config));
    *bytes = plan.config.source_mode != TEUK_B200_SOURCE_DISABLED
                 ? teuk_b200::nodal_footprint_bytes(plan)
                 : linear_footprint(plan);
  });
}

namespace {
void nodal_instance(const teuk_b200_batch& b, const int instance) {
  if (instance < 0 || instance >= b.nodal->replicas()) {
    throw std::out_of_range("batch instance index is out of range");
  }
}
}  // namespace

int teuk_b200_batch_create_with_options(const teuk_b200_config* configs,
                                        int count,
                                        const teuk_b200_batch_options* options,
                                        teuk_b200_batch** out) {
  return guarded([&] {
    require(configs != nullptr && out != nullptr && count > 0,
            "null argument or empty batch");
    const teuk_b200_batch_options opts = checked_options(options);
    std::vector<teuk_b200::Config> list;
    for (int i = 0; i < count; ++i) {
      list.push_back(teuk_b200::to_config(configs[i]));
    }
    auto b = std::make_unique<teuk_b200_batch>();
    size_t second = 0;
    for (const auto& c : list) second += c.source_mode != TEUK_B200_SOURCE_DISABLED;
    if (second > 0) {
      // validated like every pipeline first, then packed as replicas
      const teuk_b200::InstancePlan plan = teuk_b200::build_instance_plan(list[0]);
      const std::string key = nodal_group_key(list[0], opts.precision, 0.0);
      bool same = second == list.size();
      for (const auto& c : list) {
        teuk_b200::build_instance_plan(c);
        same = same && nodal_group_key(c, opts.precision, 0.0) == key;
      }
      if (!same || list[0].source_mode != TEUK_B200_SOURCE_UNRESTRICTED ||
          list[0].source_start_time != 0.0) {
        throw teuk_b200::Unsupported(
            "a batch of second-order solves needs identical configurations "
            "with the Unrestricted source from t = 0; other second-order "
            "solves run through teuk_b200_create (one nodal pipeline each)");
      }
      require_device();
      b->nodal = std::make_unique<teuk_b200::NodalPipeline>(
          plan, opts.precision, static_cast<int>(list.size()));
      b->nodal->reset_activation();
      *out = b.release();
      return;
    }
    b->batch = std::make_unique<Batch>();
    b->batch->options = opts;
    b->batch->build(list);
    *out = b.release();
  });
}

int teuk_b200_batch_create(const teuk_b200_config* configs, int count,
                           teuk_b200_batch** out) {
  return teuk_b200_batch_create_with_options(configs, count, nullptr, out);
}

int teuk_b200_batch_strip_rows(const teuk_b200_batch* b, int* rows,
                               int capacity, int* count) {
  return guarded([&] {
    require(b != nullptr && count != nullptr && capacity >= 0 &&
                (rows != nullptr || capacity == 0),
            "null argument");
    static const std::vector<int> none;
    const auto& v = b->batch ? b->batch->group_strip_rows : none;
    const int n = std::min(capacity, static_cast<int>(v.size()));
    for (int i = 0; i < n; ++i) rows[i] = v[static_cast<size_t>(i)];
    *count = static_cast<int>(v.size());
  });
}

int teuk_b200_batch_destroy(teuk_b200_batch* batch) {
  delete batch;
  return TEUK_B200_OK;
}

int teuk_b200_batch_size(const teuk_b200_batch* b, int* count) {
  return guarded([&] {
    require(b != nullptr && count != nullptr, "null argument");
    *count = b->nodal ? b->nodal->replicas()
                      : static_cast<int>(b->batch->plans.size());
  });
}

int teuk_b200_batch_shape(const teuk_b200_batch* b, int instance,
                          size_t shape[4]) {
  return guarded([&] {
    require(b != nullptr && shape != nullptr, "null argument");
    if (b->nodal) {
      nodal_instance(*b, instance);
      fill_shape(b->nodal->plan(), shape);
      return;
    }
    b->batch->check_instance(instance);
    fill_shape(b->batch->plans[static_cast<size_t>(instance)], shape);
  });
}

int teuk_b200_batch_set_state(teuk_b200_batch* b, int instance,
                              const double* state, size_t count, int memory) {
  return guarded([&] {
    require(b != nullptr, "null batch");
    if (b->nodal) {
      nodal_instance(*b, instance);
      require(count == b->nodal->plan().value_count(),
              "state complex count does not match shape");
      require(state != nullptr, "null state pointer");
      b->nodal->set_replica_state(instance, state, memory);
      return;
    }
    b->batch->set_state(instance, state, count, memory);
  });
}

int teuk_b200_batch_get_state(teuk_b200_batch* b, int instance,
                              double* state, size_t count, int memory) {
  return guarded([&] {
    require(b != nullptr, "null batch");
    if (b->nodal) {
      nodal_instance(*b, instance);
      require(count == b->nodal->plan().value_count(),
              "state complex count does not match shape");
      require(state != nullptr, "null state pointer");
      b->nodal->get_replica_state(instance, state, memory);
      return;
    }
    b->batch->get_state(instance, state, count, memory);
  });
}

int teuk_b200_batch_initialize_gaussian(teuk_b200_batch* b, int instance,
                                        const teuk_b200_gaussian* pulse) {
  return guarded([&] {
    require(b != nullptr, "null batch");
    if (b->nodal) {
      nodal_instance(*b, instance);
      initialize_nodal_gaussian(*b->nodal, pulse, instance);
      return;
    }
    initialize_gaussian(*b->batch, instance, pulse);
  });
}

int teuk_b200_batch_step(teuk_b200_batch* b, const double* dt, int steps,
                         int graph) {
  return guarded([&] {
    require(b != nullptr && dt != nullptr, "null argument");
    if (b->nodal) {
      require(steps >= 0, "step count must be nonnegative");
      const int n = b->nodal->replicas();
      for (int i = 1; i < n; ++i) {
        require(dt[i] == dt[0], "replicated second-order solves share one time step");
      }
      for (int s = 0; s < steps; ++s) {
        b->nodal->step(b->time, dt[0]);
        b->time += dt[0];
      }
      teuk_b200::check(cudaStreamSynchronize(b->nodal->stream()), "step");
      return;
    }
    std::vector<double> list(dt, dt + b->batch->plans.size());
    b->batch->step(list, steps, graph != 0);
  });
}

int teuk_b200_batch_sample_endpoint(teuk_b200_batch* b, int instance,
                                    teuk_b200_waveform_record* out,
                                    size_t capacity, size_t* count) {
  return guarded([&] {
    require(b != nullptr, "null batch");
    if (b->nodal) {
      nodal_instance(*b, instance);
      sample_nodal_endpoint(*b->nodal, out, capacity, count, instance);
      return;
    }
    b->batch->sample_endpoint(instance, out, capacity, count);
  });
}

int teuk_b200_batch_endpoint_modal(teuk_b200_batch* b, double* out,
                                   size_t capacity, size_t* count,
                                   int memory) {
  return guarded([&] {
    require(b != nullptr, "null batch");
    if (b->nodal) {
      throw teuk_b200::Unsupported(
          "band endpoint coefficients exist for linear batches only");
    }
    b->batch->endpoint_modal(out, capacity, count, memory);
  });
}

int teuk_b200_batch_set_stream(teuk_b200_batch* b, void* cuda_stream) {
  return guarded([&] {
    require(b != nullptr, "null batch");
    if (b->nodal) {
      b->nodal->set_stream(static_cast<cudaStream_t>(cuda_stream));
      return;
    }
    b->batch->stream = cuda_stream != nullptr
                           ? static_cast<cudaStream_t>(cuda_stream)
                           : b->batch->own_stream;
  });
}

int teuk_b200_batch_synchronize(teuk_b200_batch* b) {
  return guarded([&] {
    require(b != nullptr, "null batch");
    if (b->nodal) {
      teuk_b200::check(cudaStreamSynchronize(b->nodal->stream()), "synchronize");
      return;
    }
    teuk_b200::check(cudaStreamSynchronize(b->batch->stream), "synchronize");
    b->batch->check_kernel_error();
  });
}

int teuk_b200_batch_launches_per_step(const teuk_b200_batch* b,
                                      int* launches) {
  return guarded([&] {
    require(b != nullptr && launches != nullptr, "null argument");
    if (b->nodal) {
      throw teuk_b200::Unsupported(
          "a second-order batch steps through its nodal stage graph");
    }
    *launches = 4 * static_cast<int>(b->batch->groups.size());
  });
}

int teuk_b200_batch_stage_kernels(const teuk_b200_batch* b,
                                  int* streaming_groups, int* tile_groups) {
  return guarded([&] {
    require(b != nullptr && streaming_groups != nullptr &&
                tile_groups != nullptr,
            "null argument");
    if (b->nodal) {
      *streaming_groups = 0;
      *tile_groups = 0;
      return;
    }
    int streaming = 0;
    for (const teuk_b200::StageLaunch& g : b->batch->groups) {
      if (g.strips != nullptr && g.strip_count > 0) ++streaming;
    }
    *streaming_groups = streaming;
    *tile_groups = static_cast<int>(b->batch->groups.size()) - streaming;
  });
}

struct teuk_b200_server {
  std::unique_ptr<Server> server;
};

int teuk_b200_server_create(const teuk_b200_server_options* options,
                            teuk_b200_server** out) {
  return guarded([&] {
    require(options != nullptr && out != nullptr, "null argument");
    auto s = std::make_unique<teuk_b200_server>();
    s->server = std::make_unique<Server>(*options);
    *out = s.release();
  });
}

int teuk_b200_server_destroy(teuk_b200_server* server) {
  delete server;
  return TEUK_B200_OK;
}

int teuk_b200_server_submit(teuk_b200_server* server,
                            const teuk_b200_config* config,
                            const teuk_b200_gaussian* pulse, double dt,
                            int steps, uint64_t* id) {
  return guarded([&] {
    require(server != nullptr && config != nullptr && pulse != nullptr &&
                id != nullptr,
            "null argument");
    *id = server->server->submit(*config, *pulse, dt, steps);
  });
}

int teuk_b200_server_advance(teuk_b200_server* server, int steps,
                             int* active) {
  return guarded([&] {
    require(server != nullptr, "null server");
    const int n = server->server->advance(steps);
    if (active != nullptr) *active = n;
  });
}

int teuk_b200_server_result(teuk_b200_server* server, uint64_t id,
                            teuk_b200_waveform_record* out, size_t capacity,
                            size_t* count, double* latency_seconds) {
  return guarded([&] {
    require(server != nullptr, "null server");
    const ServerRequest& r = server->server->result(id);
    if (count != nullptr) *count = r.records.size();
    if (latency_seconds != nullptr) {
      *latency_seconds = r.finish_time - r.submit_time;
    }
    if (out == nullptr) return;
    require(capacity >= r.records.size(),
            "waveform record capacity is too small");
    std::copy(r.records.begin(), r.records.end(), out);
  });
}

int teuk_b200_server_stats_get(const teuk_b200_server* server,
                               teuk_b200_server_stats* out) {
  return guarded([&] {
    require(server != nullptr && out != nullptr, "null argument");
    *out = server->server->stats();
  });
}

}  // extern "C"
