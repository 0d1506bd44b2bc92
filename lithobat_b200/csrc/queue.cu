// Uneven batches in one persistent launch: the coherent passes of every
// wide-pupil size group drained from one device work queue.
//
// An uneven batch (clips of several grid sides, expose/aerial_image.py:502-548
// called once per clip in the reference) is grouped by grid side; every group
// has its own plan. The coherent transforms of the wide engine (wide.cu: one
// L x L transform per source point and field component, L = 128 .. 1024) are
// most of the work, and as per-group launch sequences they leave the GPU
// partly idle at every launch tail and round-trip their intermediate through
// HBM. Here they run as one persistent kernel over a task list built on the
// host (litho_uneven_schedule):
//
//   pass A task (group, jobs [first, first + count) of a chunk): for every
//       transform of those jobs and every spectral row ky of the band, the
//       inverse L-point FFT over kx of P M -> U[t][ky][u] in the chunk's T slot
//       (rows of the pupil table and of the mask band are read contiguously);
//   pass B task (group, item, row blocks): for every transform of the item
//       and every column u of the block, the inverse FFT over ky of U[t][.][u]
//       and J^T(u, v) += w |e|^2 in registers -> the item's partial (written once:
//       a chunk always holds whole items).
//
// Chunks of items own one of a few T slots; a slot holds enough transforms
// to keep every resident block busy while the next chunk's pass A runs (the
// slot size, slots in flight and task sizes are tunable per group).
// Each task carries the counter it waits on and the counter it adds one to
// when done: the B tasks of a chunk wait for all its A tasks; the A tasks of a
// chunk that reuses a slot wait for all B tasks of the slot's previous chunk.
// Thread blocks take tasks in list order (one atomic per task) and every
// dependency points to an earlier task, so the lowest unfinished task can
// always run: the queue cannot deadlock, whatever the number of resident
// blocks. Every wait is bounded (the library's wait limit); a wait that gives
// up records LITHO_E_TIMEOUT in the queue's status word, skips its task and
// still signals, so the launch ends.
//
// The stages before (band DFT of the masks) and after (ordered reduction,
// FFT of J, band box, synthesis, normalisation) run per group, around the
// queue launch (wide.cuh). Groups on the coarse grids of 32 / 64 points run
// their own on-chip engine first.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "fftwarp.cuh"
#include "wide.cuh"

namespace litho {

namespace {

constexpr int kQWarps = 8;
constexpr int kQMaxGroups = 8;
constexpr int kQBlocksPerSm = 2;

struct QGroup {
  const LithoJob* jobs;
  const LithoItem* items;
  const float2* table;
  const float2* mb;
  float2* T;
  float* partial;
  const float2* twL;
  int64_t slot_elems;  // complex values per T slot
  int L, h, bm, ncomp;
  int n_jobs, n_items, n_slots, slot_transforms;
};

struct QParams {
  QGroup g[kQMaxGroups];
  const LithoQueueTask* tasks;
  int n_tasks, n_groups, n_counters;
  int* head;
  int* status;
  int* counters;
};

// twiddles (L <= 1024) and the warps' transpose buffers (pass B keeps J in
// registers)
constexpr size_t kQSmem = (size_t)1024 * 8 + (size_t)kQWarps * 32 * kTbLd * 8;

__device__ __forceinline__ int ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// true once *ctr >= value, within this translation unit's wait limit
__device__ bool wait_counter(const int* ctr, int value) {
  if (ld_acquire(ctr) >= value) return true;
  const long long limit = *(volatile long long*)&g_wait_limit;
  const long long t0 = clock64();
  while (clock64() - t0 < limit) {
    __nanosleep(128);
    if (ld_acquire(ctr) >= value) return true;
  }
  return false;
}

__device__ __forceinline__ float2 ldcg2(const float2* p) { return __ldcg(p); }
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Pass A: U[t][ky][u] = sum_kx P(kx, ky) M(cx + kx, cy + ky) e^{+2 pi i kx u / L}
// for the jobs [first, first + count) of the task's chunk; a warp takes LPW
// rows ky of one transform at a time.
template <int L>
__device__ void q_pass_a(const QGroup& G, const LithoQueueTask& t, const float2* tw, float2* tb) {
  constexpr int R = L / 32, LPW = 32 / R;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int h = G.h, side = 2 * h + 1, npts = side * side, Bm = 2 * G.bm + 1, ncomp = G.ncomp;
  const int groups_per_t = (side + LPW - 1) / LPW;
  const int units = t.count * ncomp * groups_per_t;
  float2* Ts = G.T + (size_t)t.slot * G.slot_elems;
  for (int u = warp; u < units; u += kQWarps) {
    const int tc = u / groups_per_t, lg = u - tc * groups_per_t;
    const int jl = div_ncomp(tc, ncomp), c = tc - jl * ncomp;
    const int jj = t.first + jl;
    const LithoJob job = G.jobs[jj];
    if (c >= job.ncomp) continue;
    const float2* tp = G.table + ((size_t)job.tab * ncomp + c) * npts;
    const float2* m = G.mb + (size_t)job.clip * Bm * Bm;
    if (u + kQWarps < units) {   // the next unit's pupil and mask rows towards L2
      const int tc2 = (u + kQWarps) / groups_per_t, lg2 = u + kQWarps - tc2 * groups_per_t;
      const int jl2 = div_ncomp(tc2, ncomp), c2 = tc2 - jl2 * ncomp;
      const LithoJob j2 = G.jobs[t.first + jl2];
      const float2* tp2 = G.table + ((size_t)j2.tab * ncomp + c2) * npts;
      const float2* m2 = G.mb + (size_t)j2.clip * Bm * Bm;
#pragma unroll
      for (int l = 0; l < LPW; ++l) {
        const int kyi = lg2 * LPW + l, my = j2.cy + (kyi - h) + G.bm;
        if (kyi >= side || my < 0 || my >= Bm) continue;
        for (int kx = lane * 8 - h; kx <= h; kx += 256) {   // one prefetch per 64-byte piece of the rows
          prefetch_l2(tp2 + kyi * side + kx + h);
          const int mx = j2.cx + kx + G.bm;
          if (mx >= 0 && mx < Bm) prefetch_l2(m2 + (size_t)my * Bm + mx);
        }
      }
    }
    float2 x[32];
#pragma unroll
    for (int l = 0; l < LPW; ++l) {
      const int kyi = lg * LPW + l;
      const int my = job.cy + (kyi - h) + G.bm;
      const bool row_ok = kyi < side && my >= 0 && my < Bm;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int i = lane + 32 * q;
        const int kx = i <= h ? i : i - L;  // in [-h, h] when i <= h or i >= L - h
        const int mx = job.cx + kx + G.bm;
        float2 v = make_float2(0.f, 0.f);
        if (row_ok && (i <= h || i >= L - h) && mx >= 0 && mx < Bm)
          v = cmul(__ldg(tp + kyi * side + kx + h), __ldg(m + (size_t)my * Bm + mx));
        x[l * R + q] = v;
      }
    }
    warp_fft_lines<L, +1>(x, tb, tw);
    const int kyi = lg * LPW + lane / R;
    if (kyi < side) {
      float2* dst = Ts + ((size_t)((jj - t.base) * ncomp + c) * side + kyi) * L + lane % R;
#pragma unroll
      for (int s = 0; s < 32; ++s) dst[R * s] = x[s];
    }
  }
}

// Pass B: for the item's transforms and the columns u of row blocks
// [t.count, t.count + t.rows), e(u, v) = sum_ky U[t][ky][u] e^{+2 pi i ky v / L}
// and J^T(u, v) = sum_t w_t |e_t(u, v)|^2 -> partial[item][u][v].
template <int L>
__device__ void q_pass_b(const QGroup& G, const LithoQueueTask& t, const float2* tw, float2* tb) {
  constexpr int R = L / 32, LPW = 32 / R;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int h = G.h, side = 2 * h + 1, ncomp = G.ncomp;
  const LithoItem it = G.items[t.first];
  const float2* Ts = G.T + (size_t)t.slot * G.slot_elems;
  const int jb = it.job_begin, nt = (it.job_end - jb) * ncomp;
  // T rows of transform k of row block rb for this lane's registers
  auto rows_of = [&](int rb, int k) -> const float2* {
    return Ts + (size_t)((jb - t.base) * ncomp + k) * side * L + (rb * kQWarps + warp) * LPW;
  };
  for (int rb = t.count; rb < t.count + t.rows; ++rb) {
    const int u0 = (rb * kQWarps + warp) * LPW;
    float Jr[32];   // this lane's J values, in registers across the item's transforms
#pragma unroll
    for (int s = 0; s < 32; ++s) Jr[s] = 0.f;
    for (int k = 0; k < nt; ++k) {
      const int jl = div_ncomp(k, ncomp), c = k - jl * ncomp;
      const LithoJob job = G.jobs[jb + jl];
      if (c >= job.ncomp) continue;
      const float w = (float)job.weight;
      const float2* Tt = rows_of(rb, k);
      // the next transform's rows (or the next row block's first) towards L2
      // while this one is transformed
      const bool more = k + 1 < nt || rb + 1 < t.count + t.rows;
      const float2* Tn = k + 1 < nt ? rows_of(rb, k + 1) : rows_of(rb + 1, 0);
      float2 x[32];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int i = lane + 32 * q;
        const int ky = i <= h ? i : i - L;
        const bool ok = i <= h || i >= L - h;
        const float2* src = Tt + (size_t)(ky + h) * L;
        if constexpr (LPW % 2 == 0) {
#pragma unroll
          for (int l = 0; l < LPW; l += 2) {
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (ok) v = __ldcg(reinterpret_cast<const float4*>(src + l));
            x[l * R + q] = make_float2(v.x, v.y);
            x[(l + 1) * R + q] = make_float2(v.z, v.w);
          }
        } else {
          x[q] = ok ? ldcg2(src) : make_float2(0.f, 0.f);
        }
        if (ok && more) prefetch_l2(Tn + (size_t)(ky + h) * L);
      }
      warp_fft_lines<L, +1>(x, tb, tw);
#pragma unroll
      for (int s = 0; s < 32; ++s) Jr[s] = fmaf(w, cabs2(x[s]), Jr[s]);
    }
    float* pj = G.partial + ((size_t)t.first * L + u0 + lane / R) * L + lane % R;
#pragma unroll
    for (int s = 0; s < 32; ++s) pj[R * s] = Jr[s];
  }
}

// A task the kernel can run safely: every index inside its group's buffers.
__device__ bool task_ok(const QParams& P, const LithoQueueTask& t) {
  if (t.group < 0 || t.group >= P.n_groups || t.done_ctr < 0 || t.done_ctr >= P.n_counters ||
      t.wait_ctr >= P.n_counters)
    return false;
  const QGroup& G = P.g[t.group];
  if (t.slot < 0 || t.slot >= G.n_slots || t.base < 0) return false;
  const int cap = G.slot_transforms / G.ncomp;  // jobs a slot holds
  if (t.kind == 0) return t.first >= t.base && t.count >= 1 && t.first + t.count <= G.n_jobs &&
                          t.first + t.count - t.base <= cap;
  if (t.kind != 1 || t.first < 0 || t.first >= G.n_items) return false;
  const int row_blocks = G.L * G.L / 8192;
  if (t.count < 0 || t.rows < 1 || t.count + t.rows > row_blocks) return false;
  const LithoItem it = G.items[t.first];
  return it.job_begin >= t.base && it.job_end <= G.n_jobs && it.job_end - t.base <= cap &&
         it.job_begin < it.job_end;
}

template <int L>
__device__ __forceinline__ void q_run(const QGroup& G, const LithoQueueTask& t, const float2* tw, float2* tb) {
  if (t.kind == 0) q_pass_a<L>(G, t, tw, tb);
  else q_pass_b<L>(G, t, tw, tb);
}

__global__ void __launch_bounds__(kQWarps * 32, kQBlocksPerSm) k_uneven_queue(const __grid_constant__ QParams P) {
  extern __shared__ __align__(16) float2 qsm[];
  __shared__ int s_task, s_ok;
  const int warp = threadIdx.x >> 5;
  float2* tw = qsm;
  float2* tb = qsm + 1024 + warp * 32 * kTbLd;
  int tw_group = -1;
  for (;;) {
    if (threadIdx.x == 0) s_task = atomicAdd(P.head, 1);
    __syncthreads();
    const int k = s_task;
    if (k >= P.n_tasks) break;
    const LithoQueueTask t = P.tasks[k];
    if (threadIdx.x == 0) {
      bool ok = task_ok(P, t);
      if (!ok) atomicExch(P.status, LITHO_E_BAND);
      else if (t.wait_ctr >= 0 && !wait_counter(P.counters + t.wait_ctr, t.wait_value)) {
        atomicExch(P.status, LITHO_E_TIMEOUT);
        ok = false;
      }
      s_ok = ok;
    }
    __syncthreads();
    if (s_ok) {
      const QGroup& G = P.g[t.group];
      if (t.group != tw_group) {
        fill_lane_twiddles(tw, G.L, G.twL, 1);
        tw_group = t.group;
        __syncthreads();
      }
      switch (G.L) {
        case 128: q_run<128>(G, t, tw, tb); break;
        case 256: q_run<256>(G, t, tw, tb); break;
        case 512: q_run<512>(G, t, tw, tb); break;
        case 1024: q_run<1024>(G, t, tw, tb); break;
        default: break;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && t.done_ctr >= 0 && t.done_ctr < P.n_counters) {
      __threadfence();
      atomicAdd(P.counters + t.done_ctr, 1);
    }
  }
}

}  // namespace

cudaError_t set_wait_limit_queue(long long cycles) { return set_wait_limit_here(cycles); }

// ---------------------------------------------------------------------------
// host side: the schedule and the launch
// ---------------------------------------------------------------------------
namespace {

struct QChunk {
  int item0, item1, job0, job1;
};

struct QPlan {
  int lpw, side, groups_per_t, row_blocks, slot_transforms, n_slots, a_jobs, b_rows;
  std::vector<QChunk> chunks;
};

bool q_wide(const LithoAbbePlan& p) { return p.L > 64; }

// The chunks of items (each within the slot target, at least one item) and
// the resolved task sizes of one wide group. Returns a LITHO_E_* code.
int q_plan(const LithoUnevenGroup& g, QPlan& q) {
  const LithoAbbePlan& p = g.plan;
  if (!wide_plan_ok(p)) return LITHO_E_UNSUPPORTED;
  if (p.n_items < 1 || p.n_jobs < 1 || (p.ncomp_max != 1 && p.ncomp_max != 3)) return LITHO_E_SIZE;
  if (!g.blob_host) return LITHO_E_NULL;
  if (g.slot_kib < 0 || g.n_slots < 0 || g.n_slots == 1 || g.a_units < 0 || g.b_rows < 0) return LITHO_E_SIZE;
  const LithoItem* items = reinterpret_cast<const LithoItem*>(static_cast<const char*>(g.blob_host) + p.off_items);
  q.side = 2 * p.h + 1;
  q.lpw = 1024 / p.L;
  q.groups_per_t = (q.side + q.lpw - 1) / q.lpw;
  q.row_blocks = p.L / (kQWarps * q.lpw);
  const int64_t t_bytes = (int64_t)q.side * p.L * 8;           // one transform's U
  // default slot: 16 transforms per resident block (a chunk in flight keeps
  // every block busy), within [16 MiB, 1 GiB]
  int64_t target = (int64_t)g.slot_kib * 1024;
  if (!g.slot_kib) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) {
      cudaGetLastError();
      sms = 148;
    }
    target = std::min<int64_t>(std::max<int64_t>((int64_t)16 * kQBlocksPerSm * sms * t_bytes, (int64_t)16 << 20),
                               (int64_t)1 << 30);
  }
  q.n_slots = g.n_slots ? g.n_slots : 2;
  const int a_units = g.a_units ? g.a_units : 96;
  q.a_jobs = std::max(1, a_units / (p.ncomp_max * q.groups_per_t));
  q.b_rows = std::min(q.row_blocks, g.b_rows ? g.b_rows : (p.L == 128 ? 2 : 1));
  q.chunks.clear();
  q.slot_transforms = 0;
  int prev_end = 0;
  for (int i = 0; i < p.n_items; ++i) {
    const LithoItem& it = items[i];
    if (it.job_begin != prev_end || it.job_end <= it.job_begin || it.job_end > p.n_jobs) return LITHO_E_BAND;
    prev_end = it.job_end;
    const int64_t add = (int64_t)(it.job_end - it.job_begin) * p.ncomp_max;
    if (!q.chunks.empty()) {
      QChunk& c = q.chunks.back();
      const int64_t have = (int64_t)(c.job1 - c.job0) * p.ncomp_max;
      if ((have + add) * t_bytes <= target) {
        c.item1 = i + 1;
        c.job1 = it.job_end;
        q.slot_transforms = std::max<int64_t>(q.slot_transforms, have + add);
        continue;
      }
    }
    q.chunks.push_back({i, i + 1, it.job_begin, it.job_end});
    q.slot_transforms = std::max<int64_t>(q.slot_transforms, add);
  }
  if (prev_end != p.n_jobs) return LITHO_E_BAND;
  return LITHO_OK;
}

int64_t q_t_bytes(const LithoAbbePlan& p, const QPlan& q) {
  return (int64_t)q.n_slots * q.slot_transforms * q.side * p.L * 8;
}

int q_check_groups(const LithoUnevenGroup* groups, int n_groups) {
  if (!groups) return LITHO_E_NULL;
  if (n_groups < 1) return LITHO_E_SIZE;
  int wide = 0;
  for (int i = 0; i < n_groups; ++i) wide += q_wide(groups[i].plan) ? 1 : 0;
  return wide > kQMaxGroups ? LITHO_E_SIZE : LITHO_OK;
}

}  // namespace
}  // namespace litho

using namespace litho;

extern "C" int litho_uneven_group_workspace(const LithoUnevenGroup* group, size_t* bytes) {
  if (!group || !bytes) return LITHO_E_NULL;
  if (!q_wide(group->plan)) return litho_abbe_workspace(&group->plan, bytes);
  QPlan q;
  const int st = q_plan(*group, q);
  if (st) return st;
  *bytes = (size_t)wide_layout(group->plan, q_t_bytes(group->plan, q)).total;
  return LITHO_OK;
}

extern "C" int litho_uneven_schedule(const LithoUnevenGroup* groups, int n_groups, LithoQueueTask* tasks,
                                     int max_tasks, int* n_tasks, int* n_counters) {
  int st = q_check_groups(groups, n_groups);
  if (st) return st;
  if (!n_tasks || !n_counters) return LITHO_E_NULL;
  // wide groups, largest coarse grid first (the smallest tasks fill the tail)
  std::vector<int> order;
  for (int i = 0; i < n_groups; ++i)
    if (q_wide(groups[i].plan)) order.push_back(i);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return groups[a].plan.L > groups[b].plan.L; });
  std::vector<LithoQueueTask> out;
  int ctr = 0;
  int qslot = 0;  // index of the group within the kernel's table (the order above)
  for (int gi : order) {
    QPlan q;
    if ((st = q_plan(groups[gi], q)) != LITHO_OK) return st;
    const LithoAbbePlan& p = groups[gi].plan;
    const LithoItem* items =
        reinterpret_cast<const LithoItem*>(static_cast<const char*>(groups[gi].blob_host) + p.off_items);
    const int nc = (int)q.chunks.size(), ns = q.n_slots, cbase = ctr;
    ctr += 2 * nc;
    std::vector<int> nA(nc), nB(nc);
    for (int c = 0; c < nc; ++c) {
      const QChunk& ch = q.chunks[c];
      nA[c] = (ch.job1 - ch.job0 + q.a_jobs - 1) / q.a_jobs;
      nB[c] = (ch.item1 - ch.item0) * ((q.row_blocks + q.b_rows - 1) / q.b_rows);
    }
    auto emit_a = [&](int c) {
      const QChunk& ch = q.chunks[c];
      for (int j = ch.job0; j < ch.job1; j += q.a_jobs) {
        LithoQueueTask t{};
        t.kind = 0;
        t.group = qslot;
        t.slot = c % ns;
        t.base = ch.job0;
        t.first = j;
        t.count = std::min(q.a_jobs, ch.job1 - j);
        t.rows = 0;
        t.wait_ctr = c >= ns ? cbase + 2 * (c - ns) + 1 : -1;
        t.wait_value = c >= ns ? nB[c - ns] : 0;
        t.done_ctr = cbase + 2 * c;
        out.push_back(t);
      }
    };
    auto emit_b = [&](int c) {
      const QChunk& ch = q.chunks[c];
      for (int i = ch.item0; i < ch.item1; ++i) {
        (void)items;
        for (int rb = 0; rb < q.row_blocks; rb += q.b_rows) {
          LithoQueueTask t{};
          t.kind = 1;
          t.group = qslot;
          t.slot = c % ns;
          t.base = ch.job0;
          t.first = i;
          t.count = rb;
          t.rows = std::min(q.b_rows, q.row_blocks - rb);
          t.wait_ctr = cbase + 2 * c;
          t.wait_value = nA[c];
          t.done_ctr = cbase + 2 * c + 1;
          out.push_back(t);
        }
      }
    };
    // A(0) .. A(ns - 2), then A(c) followed by B(c - ns + 1), then the last Bs
    for (int c = 0; c < nc; ++c) {
      emit_a(c);
      if (c >= ns - 1) emit_b(c - ns + 1);
    }
    for (int c = std::max(0, nc - ns + 1); c < nc; ++c) emit_b(c);
    ++qslot;
  }
  *n_tasks = (int)out.size();
  *n_counters = ctr;
  if (!tasks) return LITHO_OK;
  if (max_tasks < (int)out.size()) return LITHO_E_SIZE;
  std::copy(out.begin(), out.end(), tasks);
  return LITHO_OK;
}

extern "C" int litho_uneven_queue_workspace(int n_counters, size_t* bytes) {
  if (!bytes) return LITHO_E_NULL;
  if (n_counters < 0) return LITHO_E_SIZE;
  *bytes = (size_t)align16(16 + (int64_t)n_counters * 4);
  return LITHO_OK;
}

extern "C" int litho_uneven_run(const LithoUnevenGroup* groups, int n_groups, const LithoQueueTask* tasks_dev,
                                int n_tasks, int n_counters, void* queue_ws, size_t queue_ws_bytes,
                                cudaStream_t s) {
  int st = q_check_groups(groups, n_groups);
  if (st) return st;
  if (n_tasks < 0 || n_counters < 0) return LITHO_E_SIZE;
  if (n_tasks > 0 && (!tasks_dev || !queue_ws)) return LITHO_E_NULL;
  if (((uintptr_t)queue_ws & 15) || ((uintptr_t)tasks_dev & 7)) return LITHO_E_ALIGN;
  if (queue_ws && queue_ws_bytes < (size_t)align16(16 + (int64_t)n_counters * 4)) return LITHO_E_WORKSPACE;
  // every group is checked before anything is launched
  for (int i = 0; i < n_groups; ++i) {
    const LithoUnevenGroup& g = groups[i];
    if (q_wide(g.plan)) continue;
    size_t need = 0;
    if ((st = litho_abbe_workspace(&g.plan, &need)) != LITHO_OK) return st;
    if (g.ws_bytes < need) return LITHO_E_WORKSPACE;
    if (!g.blob_dev || !g.table_dev || !g.masks_dev || !g.image_dev || !g.peak_dev || !g.workspace_dev)
      return LITHO_E_NULL;
  }
  std::vector<int> order;
  for (int i = 0; i < n_groups; ++i)
    if (q_wide(groups[i].plan)) order.push_back(i);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return groups[a].plan.L > groups[b].plan.L; });
  QParams P{};
  std::vector<WideLayout> lay(order.size());
  for (size_t k = 0; k < order.size(); ++k) {
    const LithoUnevenGroup& g = groups[order[k]];
    const LithoAbbePlan& p = g.plan;
    QPlan q;
    if ((st = q_plan(g, q)) != LITHO_OK) return st;
    if (!g.blob_dev || !g.table_dev || !g.masks_dev || !g.image_dev || !g.peak_dev || !g.workspace_dev)
      return LITHO_E_NULL;
    if (((uintptr_t)g.workspace_dev & 15) || ((uintptr_t)g.blob_dev & 15) || ((uintptr_t)g.masks_dev & 7) ||
        ((uintptr_t)g.table_dev & 7))
      return LITHO_E_ALIGN;
    lay[k] = wide_layout(p, q_t_bytes(p, q));
    if ((int64_t)g.ws_bytes < lay[k].total) return LITHO_E_WORKSPACE;
    const char* b = static_cast<const char*>(g.blob_dev);
    char* w = static_cast<char*>(g.workspace_dev);
    QGroup& G = P.g[k];
    G.jobs = reinterpret_cast<const LithoJob*>(b + p.off_jobs);
    G.items = reinterpret_cast<const LithoItem*>(b + p.off_items);
    G.table = static_cast<const float2*>(g.table_dev);
    G.mb = reinterpret_cast<const float2*>(w + lay[k].mb);
    G.T = reinterpret_cast<float2*>(w + lay[k].T);
    G.partial = reinterpret_cast<float*>(w + lay[k].partial);
    G.slot_elems = (int64_t)q.slot_transforms * q.side * p.L;
    G.L = p.L;
    G.h = p.h;
    G.bm = p.bm;
    G.ncomp = p.ncomp_max;
    G.n_jobs = p.n_jobs;
    G.n_items = p.n_items;
    G.n_slots = q.n_slots;
    G.slot_transforms = q.slot_transforms;
  }
  P.n_groups = (int)order.size();
  P.n_counters = n_counters;
  if (!order.empty() && n_tasks < 1) return LITHO_E_SIZE;
  // coarse-grid groups: their own on-chip engine
  for (int i = 0; i < n_groups; ++i) {
    const LithoUnevenGroup& g = groups[i];
    if (q_wide(g.plan)) continue;
    if ((st = litho_abbe_tabled(&g.plan, g.blob_dev, g.table_dev, g.masks_dev, g.image_dev, g.peak_dev,
                                g.workspace_dev, g.ws_bytes, s)) != LITHO_OK)
      return st;
  }
  if (order.empty()) return LITHO_OK;
  // the wide groups' band DFTs, then the queue
  int sms = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (sms <= 0) sms = 148;
  for (size_t k = 0; k < order.size(); ++k) {
    const LithoUnevenGroup& g = groups[order[k]];
    if ((st = wide_prepare(g.plan, g.masks_dev, g.workspace_dev, lay[k], s, sms)) != LITHO_OK) return st;
    P.g[k].twL = twiddles_for(g.plan.L, reinterpret_cast<float2*>(static_cast<char*>(g.workspace_dev) + lay[k].twL),
                              s);
  }
  cudaError_t e;
  if (n_tasks > 0) {
    int* qw = static_cast<int*>(queue_ws);
    if ((e = cudaMemsetAsync(qw, 0, (size_t)align16(16 + (int64_t)n_counters * 4), s)) != cudaSuccess) return (int)e;
    P.tasks = tasks_dev;
    P.n_tasks = n_tasks;
    P.status = qw;
    P.head = qw + 1;
    P.counters = qw + 4;
    cudaFuncSetAttribute(k_uneven_queue, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kQSmem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_uneven_queue, kQWarps * 32, kQSmem) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    const int grid = (int)std::min<int64_t>((int64_t)sms * per_sm, n_tasks);
    k_uneven_queue<<<grid, kQWarps * 32, kQSmem, s>>>(P);
    if ((e = cudaGetLastError()) != cudaSuccess) return (int)e;
  }
  for (size_t k = 0; k < order.size(); ++k) {
    const LithoUnevenGroup& g = groups[order[k]];
    if ((st = wide_finish(g.plan, g.blob_dev, g.image_dev, g.peak_dev, g.workspace_dev, lay[k], true, s)) !=
        LITHO_OK)
      return st;
  }
  return LITHO_OK;
}

extern "C" int litho_uneven_status(const void* queue_ws, cudaStream_t s) {
  if (!queue_ws) return LITHO_E_NULL;
  int st = 0;
  cudaError_t e = cudaMemcpyAsync(&st, queue_ws, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return (int)e;
  return st;
}
