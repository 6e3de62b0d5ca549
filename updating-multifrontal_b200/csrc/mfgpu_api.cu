// C ABI (include/mfgpu.h): handle lifetime, level-by-level orchestration of the
// factor / localized update / solve / apply on one CUDA stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <chrono>
#include <map>
#include <tuple>
#include <deque>
#include <functional>
#include <condition_variable>
#include <thread>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/mfgpu.h"
#include "device.cuh"
#include "schedule.hpp"

using mfgpu::DevError;
using mfgpu::FrontDev;
using mfgpu::Schedule;
using mfgpu::SepDev;
using mfgpu::Task;

namespace {

struct CudaError : std::runtime_error {
  int status;
  CudaError(const std::string& m, int s) : std::runtime_error(m), status(s) {}
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) {
    int st = (e == cudaErrorMemoryAllocation) ? MFGPU_ERR_OOM : MFGPU_ERR_CUDA;
    throw CudaError(std::string(what) + ": " + cudaGetErrorString(e), st);
  }
}

// Host-side fault injection (mfgpu_inject_alloc_failure): the number of
// device allocations that still succeed before one is failed; -1 = disarmed.
std::atomic<long long> g_alloc_budget{-1};

// True when this allocation is the one chosen to fail (disarms the injection).
bool injectedAllocFailure() {
  long long k = g_alloc_budget.load();
  while (k >= 0) {
    if (g_alloc_budget.compare_exchange_weak(k, k - 1)) return k == 0;
  }
  return false;
}

template <class T>
T* dalloc(size_t count, const char* what) {
  void* p = nullptr;
  if (count == 0) count = 1;
  if (injectedAllocFailure())
    throw CudaError(std::string(what) + ": injected device allocation failure", MFGPU_ERR_OOM);
  ck(cudaMalloc(&p, count * sizeof(T)), what);
  return static_cast<T*>(p);
}

int64_t tilesOf(const Task& t) {
  const int64_t a = (t.rows + mfgpu::kTaskTile - 1) / mfgpu::kTaskTile;
  const int64_t b = (t.cols + mfgpu::kTaskTile - 1) / mfgpu::kTaskTile;
  return a * b;
}

// A group of tasks executed by one launch.
struct Group {
  int64_t task0 = 0, ntasks = 0, pref0 = 0, ntiles = 0;
};

// Everything one factorization pass needs: per level the fronts and separators
// to (re)compute and their task groups, all in one device buffer.
struct Plan {
  struct Level {
    int64_t f0 = 0, nf = 0, s0 = 0, ns = 0;  // offsets into the id list
    int maxN = 0, maxn = 0;
    Group ftask, sbase, sadd0, sadd1;
    int64_t cpref0 = 0;   // offset of the cooperative kernel's phase prefixes in cpref
    int coopItems = 0;    // largest work-item count of any cooperative phase
    int coopOuter = 0;    // outer panel width the phase prefixes were built with (0: default)
    // A batch plan (several problems' fronts in one plan, the serving loop's)
    // factors a level's fronts in consecutive partitions, each with the kernel
    // its problems would get alone: `subs` holds them (f0, nf, maxN, maxn,
    // cpref0, coopItems, coopOuter of a partition, its kernel in `kind`).
    // Empty: one partition, the level itself, kernel by the size rules.
    struct Sub;
    std::vector<Sub> subs;
  };
  size_t tcPackBytes = 0;   // largest tensor-core panel pack any level of the plan needs
  std::vector<Level> lv;
  std::vector<int> real;    // batch plans: the schedule's front id of each entry of `ids`
  std::vector<Task> tasks;
  std::vector<int64_t> pref;
  std::vector<int> ids;
  std::vector<int> cpref;
  int nfronts = 0;
  double flops = 0;
  // device copies
  Task* d_tasks = nullptr;
  int64_t* d_pref = nullptr;
  int* d_ids = nullptr;
  int* d_cpref = nullptr;
  size_t cap_tasks = 0, cap_pref = 0, cap_ids = 0, cap_cpref = 0;

  void release() {
    cudaFree(d_tasks);
    cudaFree(d_pref);
    cudaFree(d_ids);
    cudaFree(d_cpref);
    d_tasks = nullptr;
    d_pref = nullptr;
    d_ids = nullptr;
    d_cpref = nullptr;
    cap_tasks = cap_pref = cap_ids = cap_cpref = 0;
  }

  // A group is built by beginGroup, appendGroup (the tasks of some owners,
  // optionally rewritten by fx), endGroup.
  Group beginGroup() {
    Group g;
    g.task0 = (int64_t)tasks.size();
    g.pref0 = (int64_t)pref.size();
    pref.push_back(0);
    return g;
  }
  void appendGroup(Group& g, const std::vector<Task>& src, const std::vector<int64_t>& ptr,
                   const std::vector<int>& owners, int pick /* -1 all, 0/1 add task k */,
                   const std::function<void(Task&)>& fx = nullptr) {
    int64_t acc = pref.back();
    for (int o : owners) {
      int64_t a, b;
      if (pick < 0) {
        a = ptr[o];
        b = ptr[o + 1];
      } else {
        a = 2 * (int64_t)o + pick;
        b = a + 1;
      }
      for (int64_t t = a; t < b; t++) {
        tasks.push_back(src[t]);
        if (fx) fx(tasks.back());
        acc += tilesOf(src[t]);
        pref.push_back(acc);
      }
    }
    (void)g;
  }
  void endGroup(Group& g) {
    g.ntasks = (int64_t)tasks.size() - g.task0;
    g.ntiles = pref.back();
    if (g.ntasks == 0) pref.pop_back();
  }
  Group addGroup(const std::vector<Task>& src, const std::vector<int64_t>& ptr,
                 const std::vector<int>& owners, int pick) {
    Group g = beginGroup();
    appendGroup(g, src, ptr, owners, pick);
    endGroup(g);
    return g;
  }

  void upload(cudaStream_t st) {
    auto grow = [](auto*& p, size_t& cap, size_t need, const char* what) {
      if (need <= cap) return;
      cudaFree(p);
      p = nullptr;
      using T = std::remove_reference_t<decltype(*p)>;
      size_t c = std::max(need, cap * 2);
      p = dalloc<T>(c, what);
      cap = c;
    };
    grow(d_tasks, cap_tasks, tasks.size(), "alloc plan tasks");
    grow(d_pref, cap_pref, pref.size(), "alloc plan prefixes");
    grow(d_ids, cap_ids, ids.size(), "alloc plan ids");
    grow(d_cpref, cap_cpref, cpref.size(), "alloc plan phase prefixes");
    if (!tasks.empty())
      ck(cudaMemcpyAsync(d_tasks, tasks.data(), tasks.size() * sizeof(Task), cudaMemcpyHostToDevice, st),
         "upload tasks");
    if (!pref.empty())
      ck(cudaMemcpyAsync(d_pref, pref.data(), pref.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st),
         "upload prefixes");
    if (!ids.empty())
      ck(cudaMemcpyAsync(d_ids, ids.data(), ids.size() * sizeof(int), cudaMemcpyHostToDevice, st),
         "upload ids");
    if (!cpref.empty())
      ck(cudaMemcpyAsync(d_cpref, cpref.data(), cpref.size() * sizeof(int), cudaMemcpyHostToDevice,
                         st),
         "upload phase prefixes");
    // host vectors must outlive the async copies
    ck(cudaStreamSynchronize(st), "plan upload");
  }
};

struct Plan::Level::Sub {
  int64_t f0 = 0, nf = 0;
  int maxN = 0, maxn = 0;
  int64_t cpref0 = 0;
  int coopItems = 0, coopOuter = 0;
  int kind = -1;
};

// Optional per-kernel-class device timing: an event pair around each launch
// group, read back after the call's final synchronisation.
struct Profiler {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  struct Mark {
    int cls;
    cudaEvent_t a, b;
    int level;
  };
  bool verbose = false;   // MFGPU_VERBOSE=1: one stderr line per launch group
  int level = -1;         // level tag of the next marks
  std::vector<Mark> marks;
  int64_t launches[MFGPU_KC_COUNT] = {};
  double ms[MFGPU_KC_COUNT] = {};
  double flops[MFGPU_KC_COUNT] = {};
  double bytes[MFGPU_KC_COUNT] = {};

  cudaEvent_t ev() {
    if (used == pool.size()) {
      cudaEvent_t e;
      ck(cudaEventCreate(&e), "profiler event");
      pool.push_back(e);
    }
    return pool[used++];
  }
  void begin(int cls, cudaStream_t st) {
    if (!on) return;
    Mark m{cls, ev(), nullptr, level};
    ck(cudaEventRecord(m.a, st), "profiler record");
    marks.push_back(m);
  }
  void end(cudaStream_t st) {
    if (!on || marks.empty()) return;
    marks.back().b = ev();
    ck(cudaEventRecord(marks.back().b, st), "profiler record");
  }
  void collect() {
    for (const Mark& m : marks) {
      float t = 0;
      if (m.b && cudaEventElapsedTime(&t, m.a, m.b) == cudaSuccess) {
        ms[m.cls] += t;
        launches[m.cls] += 1;
        if (verbose) fprintf(stderr, "[mfgpu] class %d level %d %.3f ms\n", m.cls, m.level, t);
      }
    }
    marks.clear();
    used = 0;
  }
  void reset() {
    marks.clear();
    used = 0;
    for (int i = 0; i < MFGPU_KC_COUNT; i++) launches[i] = 0, ms[i] = flops[i] = bytes[i] = 0;
  }
  ~Profiler() {
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
};

}  // namespace

struct mfgpu_handle {
  std::shared_ptr<Schedule> S;   // shared with the serving loop's views
  mfgpu_options opt{};
  int device = 0;
  cudaStream_t own = nullptr, stream = nullptr;
  std::string err;
  mfgpu_stats stats{};
  bool factored = false;
  int n = 0;
  int64_t nnz = 0;
  std::vector<int> h_rowptr, h_colind;

  void* d_F = nullptr;             // front arena (double or float)
  void* d_Sep = nullptr;           // separator arena (double or float)
  double* d_val = nullptr;
  int* d_rp = nullptr;
  int* d_ci = nullptr;
  int* d_dofs = nullptr;
  FrontDev* d_fr = nullptr;
  SepDev* d_sp = nullptr;
  int64_t* d_woff = nullptr;
  DevError* d_err = nullptr;
  unsigned waitLimit = 0;          // poll limit of the bounded device waits (0: built-in), kept in d_err
  // CUDA graphs: the full factorization's level schedule and the solve sweeps
  // (FP64) / preconditioner applications (mixed) per right-hand-side buffer
  // and count, captured once their launches have run eagerly and replayed
  // with one cudaGraphLaunch.  MFGPU_GRAPHS=0 turns them off; a capture the
  // runtime refuses turns them off for the handle.
  bool graphs = true;
  int fullRuns = 0;
  cudaGraphExec_t fullGraph = nullptr;
  std::map<std::tuple<const void*, const void*, int>, cudaGraphExec_t> sweepGraphs;
  std::map<std::tuple<const void*, const void*, int>, int> sweepSeen;
  void* d_slots = nullptr;     // diagonal-block hand-off slots of the cooperative kernel
  void* d_tcpack = nullptr;    // tensor-core panel images (mixed path)
  void* d_pslot = nullptr;     // factored diagonal blocks of the panel-by-panel kernels
  size_t tcPackCap = 0;
  unsigned* d_gbar = nullptr;  // grid-barrier arrival counter of the cooperative kernels
  // Cooperative (flag-ordered) sweeps: per level, its forward / backward task
  // lists and flag offsets in d_flow; the ready flags of one launch in d_flags.
  struct FlowLevel {
    int64_t fwd = 0, bwd = 0, flagoff = 0;
    int nfwd = 0, nbwd = 0, nflags = 0;
  };
  std::vector<FlowLevel> flow;
  int* d_flow = nullptr;       // shared with serving-loop views
  int* d_flags = nullptr;      // per handle (views have their own)
  int maxFlags = 0;
  void* d_Dinv = nullptr;      // inverses of the cooperative-sweep levels' 64 x 64 pivot blocks
  int64_t* d_dinv_off = nullptr;   // per front: element offset in d_Dinv, -1 outside those levels
  std::vector<int64_t> h_dinv_off; // host copy
  int64_t dinvElems = 0;
  // solve workspaces (d_Wd / d_Td hold elements of the factor's precision)
  double* d_Wd = nullptr;
  size_t capW = 0;
  double* d_X = nullptr;
  size_t capX = 0;
  double* d_Td = nullptr;
  size_t capT = 0;
  // mixed precision: scaling and refinement buffers
  bool mixed = false;
  int tcMinN = 4096;               // mixed: smallest level maxN run on the tensor cores (0 = never)
  int tcSplit = 3;                 // mixed: 3 = three-term TF32 products, 1 = plain TF32, 2 = BF16
  int tcSplit3Levels = -1;         // >= 0: tcSplit only on the top levels 0 .. this - 1,
  int tcSplitLow = 1;              //   tcSplitLow (plain TF32 or BF16) below them
  int tcSub = 128;                 // mixed: sub-panel width inside each 512-column outer panel of a
                                   // tensor-core level (0 or 512: no sub-panels)
  int fusedMinFronts = 148;        // fewest fronts for the one-CTA-per-front kernel
  bool subpanel = true;            // tensor-core levels: sub-panels by k_diag_factor + k_panel_trsm
                                   // (MFGPU_SUBPANEL=0: by the cooperative kernel)
  int panelMaxN = 0;               // largest front of a level factored panel by panel (0: never;
                                   // MFGPU_PANEL_MAX_N; the autotuner may still pick the kernel)
  size_t esz = sizeof(double);     // bytes per factor element
  double* d_scale = nullptr;       // s = 1/sqrt(diag(A)) of the last full factorization
  double* d_iscale = nullptr;      // 1/s
  double *d_B = nullptr, *d_R = nullptr, *d_P = nullptr, *d_Q = nullptr, *d_Z = nullptr;
  size_t capB = 0, capR = 0, capP = 0, capQ = 0, capZ = 0;
  float* d_x32 = nullptr;
  size_t cap32 = 0;
  double* d_dotp = nullptr;
  size_t capDot = 0;
  double* d_sc = nullptr;          // refinement scalars, 5 x nseg x 16
  int* d_active = nullptr;         // refinement: (segment, column) pairs still iterating
  // segments of the solution vector: the problems of a batch (one otherwise);
  // the refinement's dots, scalars and convergence test are per segment
  int nseg = 1, nchunks = 0;
  int* d_segrow = nullptr;         // nseg + 1 segment boundaries (rows)
  int* d_chunkrow = nullptr;       // nchunks + 1 dot chunk boundaries (rows)
  int* d_segchunk = nullptr;       // nseg + 1: first dot chunk of each segment
  // device stencil assembly: per-row change flags (+ a counter) and the rows found
  int* d_flag = nullptr;
  int* d_modbuf = nullptr;
  size_t capMod = 0;
  int* d_all = nullptr;      // every front id then every separator id, level order
  int64_t woffTotal = 0;     // sum over fronts of 2N
  Plan full, upd;
  std::vector<int> tuned;    // per level of the full plan: kernel picked by mfgpu_autotune, or -1
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int64_t device_bytes = 0;
  Profiler prof;
  std::vector<int> lvMaxN;   // largest front (n + m) per level
  std::vector<int> lvMaxn;   // largest pivot count per level
  int solveCoopMinN = 1024;  // levels with a front this large use the cooperative sweeps
  bool stepped = false;      // MFGPU_STEPPED=1: per-step launches instead of the cooperative kernel
  // Separator widths 2-3: the operators are nonsymmetric, every front is
  // stored whole and factored by pivoted LU (FP64), pivots in d_ipiv beside
  // each front's pivot DOFs.
  bool lu = false;
  int* d_ipiv = nullptr;
  // A view (the serving loop's per-slot handle) shares the base handle's
  // schedule, arenas, matrix pattern and tables and owns only its stream, its
  // front table, values, error word, scratch and workspaces.
  bool view = false;

  ~mfgpu_handle() {
    if (stream) cudaStreamSynchronize(stream);
    full.release();
    upd.release();
    if (!view) {
      cudaFree(d_F);
      cudaFree(d_Sep);
      cudaFree(d_rp);
      cudaFree(d_ci);
      cudaFree(d_dofs);
      cudaFree(d_sp);
      cudaFree(d_woff);
      cudaFree(d_scale);
      cudaFree(d_iscale);
      cudaFree(d_segrow);
      cudaFree(d_chunkrow);
      cudaFree(d_segchunk);
      cudaFree(d_all);
      cudaFree(d_dinv_off);
      cudaFree(d_ipiv);
      cudaFree(d_flow);
    }
    cudaFree(d_flags);
    cudaFree(d_Dinv);
    cudaFree(d_val);
    cudaFree(d_fr);
    cudaFree(d_err);
    cudaFree(d_slots);
    cudaFree(d_tcpack);
    cudaFree(d_pslot);
    cudaFree(d_gbar);
    cudaFree(d_Wd);
    cudaFree(d_X);
    cudaFree(d_Td);
    cudaFree(d_B);
    cudaFree(d_R);
    cudaFree(d_P);
    cudaFree(d_Q);
    cudaFree(d_Z);
    cudaFree(d_x32);
    cudaFree(d_dotp);
    cudaFree(d_sc);
    cudaFree(d_active);
    cudaFree(d_flag);
    cudaFree(d_modbuf);
    dropGraphs(true, true);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (own) cudaStreamDestroy(own);
  }

  // The schedule's front id of entry i of a plan's id list (batch plans list
  // per-problem front copies under their own ids).
  static int realId(const Plan& P, int64_t i) { return P.real.empty() ? P.ids[i] : P.real[i]; }

  // Build a plan for the given dirty fronts (global ids); separators adjacent
  // to a dirty front at their level are recomputed.
  void buildPlan(Plan& P, const std::vector<char>& dirtyFront) {
    const Schedule& s = *S;
    P.lv.assign(s.levels, Plan::Level());
    P.tasks.clear();
    P.pref.clear();
    P.ids.clear();
    P.real.clear();
    P.cpref.clear();
    P.nfronts = 0;
    P.flops = 0;
    P.tcPackBytes = 0;
    for (int ell = s.levels - 1; ell >= 0; ell--) {
      Plan::Level& L = P.lv[ell];
      std::vector<int> fl, sl;
      for (int b = 0; b < s.lv[ell].nbox; b++) {
        int f = s.lv[ell].front0 + b;
        if (dirtyFront[f]) fl.push_back(f);
      }
      for (int e = 0; e < s.lv[ell].nsep; e++) {
        int k = s.lv[ell].sep0 + e;
        const mfgpu::Sep& sp = s.seps[k];
        if (dirtyFront[sp.box[0]] || dirtyFront[sp.box[1]]) sl.push_back(k);
      }
      L.f0 = (int64_t)P.ids.size();
      L.nf = (int64_t)fl.size();
      P.ids.insert(P.ids.end(), fl.begin(), fl.end());
      L.s0 = (int64_t)P.ids.size();
      L.ns = (int64_t)sl.size();
      P.ids.insert(P.ids.end(), sl.begin(), sl.end());
      for (int f : fl) {
        L.maxN = std::max(L.maxN, s.fronts[f].N);
        L.maxn = std::max(L.maxn, s.fronts[f].n);
        P.flops += s.front_flops(s.fronts[f]);
      }
      P.nfronts += (int)fl.size();
      L.ftask = P.addGroup(s.front_tasks, s.front_task_ptr, fl, -1);
      L.sbase = P.addGroup(s.sep_tasks, s.sep_task_ptr, sl, -1);
      L.sadd0 = P.addGroup(s.sep_add_tasks, s.sep_task_ptr, sl, 0);
      L.sadd1 = P.addGroup(s.sep_add_tasks, s.sep_task_ptr, sl, 1);
      L.cpref0 = (int64_t)P.cpref.size();
      // phase tables for every level the cooperative kernel can take (also the
      // ones the size rules give to k_front_small: the autotuner may not)
      if (!fl.empty() && mfgpu::coop_fits((int)fl.size())) {
        std::vector<int> nn, NN;
        for (int f : fl) {
          nn.push_back(s.fronts[f].n);
          NN.push_back(s.fronts[f].N);
        }
        const int W = mfgpu::tc_outer();
        const bool tc = mixed && tcLevel(L);
        L.coopOuter = tc && tcSub > 0 && tcSub < W ? tcSub : 0;
        std::vector<int> pp = mfgpu::coop_phase_prefix(nn, NN, L.maxn, L.coopOuter);
        P.cpref.insert(P.cpref.end(), pp.begin(), pp.end());
        // the most work items any phase has: a level with little parallel work
        // runs on fewer CTAs, so its grid barriers are cheaper
        const size_t stride = fl.size() + 1;
        for (size_t q = 0; q + stride <= pp.size(); q += stride)
          L.coopItems = std::max(L.coopItems, pp[q + fl.size()]);
        if (tc) {
          const int w = L.coopOuter > 0 ? L.coopOuter : W;
          for (int K = 0; K < L.maxn; K += w)
            for (int ww : {w, W})
              if (K % ww == 0)
                P.tcPackBytes = std::max(
                    P.tcPackBytes,
                    mfgpu::tc_pack_bytes((int)fl.size(), mfgpu::tc_pack_cap(nn, NN, K, ww)));
        }
      }
    }
  }

  // One problem of a batch plan: its dirty fronts, the id base of its front
  // copies (front f is vbase + f in the plan), the rewrite of its tasks into
  // its private copies, and the element offset of its CSR values.
  struct BatchMember {
    const std::vector<char>* dirty;
    int vbase;
    std::function<void(Task&)> move;
    int64_t valoff;
  };

  // A plan over several problems that share this schedule and differ in their
  // values (the serving loop's requests): every level's assembly, kernel and
  // separator launches cover all of them; each level's fronts are grouped by
  // the kernel the size rules give each problem alone, so every front is
  // factored exactly as in a plan of its problem alone.
  void buildPlanBatch(Plan& P, const std::vector<BatchMember>& M) {
    const Schedule& s = *S;
    P.lv.assign(s.levels, Plan::Level());
    P.tasks.clear();
    P.pref.clear();
    P.ids.clear();
    P.real.clear();
    P.cpref.clear();
    P.nfronts = 0;
    P.flops = 0;
    P.tcPackBytes = 0;
    const int W = mfgpu::tc_outer();
    for (int ell = s.levels - 1; ell >= 0; ell--) {
      Plan::Level& L = P.lv[ell];
      const size_t nm = M.size();
      std::vector<std::vector<int>> fl(nm), sl(nm);
      std::vector<int> kind(nm, LK_NONE), kinds;
      for (size_t m = 0; m < nm; m++) {
        const std::vector<char>& dirty = *M[m].dirty;
        Plan::Level one;
        for (int b = 0; b < s.lv[ell].nbox; b++) {
          const int f = s.lv[ell].front0 + b;
          if (!dirty[f]) continue;
          fl[m].push_back(f);
          one.maxN = std::max(one.maxN, s.fronts[f].N);
          one.maxn = std::max(one.maxn, s.fronts[f].n);
        }
        for (int e = 0; e < s.lv[ell].nsep; e++) {
          const int k = s.lv[ell].sep0 + e;
          if (dirty[s.seps[k].box[0]] || dirty[s.seps[k].box[1]]) sl[m].push_back(k);
        }
        one.nf = (int64_t)fl[m].size();
        kind[m] = ruleKernel(one);
        if (kind[m] != LK_NONE && std::find(kinds.begin(), kinds.end(), kind[m]) == kinds.end())
          kinds.push_back(kind[m]);
      }
      L.f0 = (int64_t)P.ids.size();
      for (int kd : kinds) {
        Plan::Level::Sub u;
        u.kind = kd;
        u.f0 = (int64_t)P.ids.size();
        std::vector<int> nn, NN;
        for (size_t m = 0; m < nm; m++) {
          if (kind[m] != kd) continue;
          for (int f : fl[m]) {
            P.ids.push_back(M[m].vbase + f);
            P.real.push_back(f);
            u.maxN = std::max(u.maxN, s.fronts[f].N);
            u.maxn = std::max(u.maxn, s.fronts[f].n);
            nn.push_back(s.fronts[f].n);
            NN.push_back(s.fronts[f].N);
            P.flops += s.front_flops(s.fronts[f]);
          }
        }
        u.nf = (int64_t)P.ids.size() - u.f0;
        if (kd == LK_COOP || kd == LK_TC) {
          u.coopOuter = kd == LK_TC && tcSub > 0 && tcSub < W ? tcSub : 0;
          u.cpref0 = (int64_t)P.cpref.size();
          std::vector<int> pp = mfgpu::coop_phase_prefix(nn, NN, u.maxn, u.coopOuter);
          P.cpref.insert(P.cpref.end(), pp.begin(), pp.end());
          const size_t stride = nn.size() + 1;
          for (size_t q = 0; q + stride <= pp.size(); q += stride)
            u.coopItems = std::max(u.coopItems, pp[q + nn.size()]);
          if (kd == LK_TC) {
            const int w = u.coopOuter > 0 ? u.coopOuter : W;
            for (int K = 0; K < u.maxn; K += w)
              for (int ww : {w, W})
                if (K % ww == 0)
                  P.tcPackBytes = std::max(
                      P.tcPackBytes,
                      mfgpu::tc_pack_bytes((int)nn.size(), mfgpu::tc_pack_cap(nn, NN, K, ww)));
          }
        }
        L.maxN = std::max(L.maxN, u.maxN);
        L.maxn = std::max(L.maxn, u.maxn);
        L.subs.push_back(u);
      }
      L.nf = (int64_t)P.ids.size() - L.f0;
      P.nfronts += (int)L.nf;
      L.s0 = (int64_t)P.ids.size();
      for (size_t m = 0; m < nm; m++)
        for (int k : sl[m]) {
          P.ids.push_back(k);
          P.real.push_back(k);
        }
      L.ns = (int64_t)P.ids.size() - L.s0;
      auto group = [&](const std::vector<Task>& src, const std::vector<int64_t>& ptr,
                       const std::vector<std::vector<int>>& own, int pick) {
        Group g = P.beginGroup();
        for (size_t m = 0; m < nm; m++) {
          const BatchMember& bm = M[m];
          P.appendGroup(g, src, ptr, own[m], pick, [&bm](Task& t) {
            bm.move(t);
            if (t.kind == mfgpu::TK_SPARSE) t.src_off = bm.valoff;
          });
        }
        P.endGroup(g);
        return g;
      };
      L.ftask = group(s.front_tasks, s.front_task_ptr, fl, -1);
      L.sbase = group(s.sep_tasks, s.sep_task_ptr, sl, -1);
      L.sadd0 = group(s.sep_add_tasks, s.sep_task_ptr, sl, 0);
      L.sadd1 = group(s.sep_add_tasks, s.sep_task_ptr, sl, 1);
    }
  }

  template <class T>
  void runGroup(const Plan& P, const Group& g, int64_t bytes) {
    if (g.ntasks == 0 || g.ntiles == 0) return;
    prof.begin(MFGPU_KC_ASSEMBLE, stream);
    mfgpu::launch_tasks<T>(P.d_tasks + g.task0, P.d_pref + g.pref0, (int)g.ntasks, g.ntiles,
                           (T*)d_F, (T*)d_Sep, d_rp, d_ci, d_val, d_dofs, mixed ? d_scale : nullptr,
                           stream);
    ck(cudaGetLastError(), "launch assembly (k_tasks)");
    prof.end(stream);
    if (prof.on) prof.bytes[MFGPU_KC_ASSEMBLE] += (double)bytes;
  }

  // Bytes an assembly group must move: every destination element written,
  // plus the element read for copies and adds (read twice for adds).
  int64_t groupBytes(const Plan& P, const Group& g) const {
    if (!prof.on) return 0;
    int64_t b = 0;
    for (int64_t t = g.task0; t < g.task0 + g.ntasks; t++) {
      const Task& T = P.tasks[t];
      int64_t e = T.lower ? (int64_t)T.rows * (T.rows + 1) / 2 : (int64_t)T.rows * T.cols;
      int mult = T.kind == mfgpu::TK_ZERO ? 1 : T.kind == mfgpu::TK_ADD ? 3 : 2;
      b += e * (int64_t)esz * mult;
    }
    return b;
  }

  // Level kernels.  The size rules choose one per level; mfgpu_autotune can
  // replace the choice for the levels of the full factorization by timing.
  enum LevelKernel { LK_NONE = -1, LK_FUSED = 0, LK_COOP = 1, LK_TC = 2, LK_STEPPED = 3, LK_LU = 4,
                     LK_PANEL = 5 };

  int ruleKernel(const Plan::Level& L) const {
    if (L.nf <= 0) return LK_NONE;
    if (lu) return LK_LU;
    if (useFused((int)L.nf, L.maxN)) return LK_FUSED;
    if (!mfgpu::coop_fits((int)L.nf) || (stepped && !mixed)) return LK_STEPPED;
    if (mixed && tcLevel(L)) return LK_TC;
    if (panelFits(L)) return LK_PANEL;
    return LK_COOP;
  }

  int levelKernel(const Plan& P, const Plan::Level& L, int ell) const {
    if (&P == &full && ell < (int)tuned.size() && tuned[ell] != LK_NONE && L.nf > 0)
      return tuned[ell];
    return ruleKernel(L);
  }

  // Levels of moderate fronts (up to panelMaxN) go panel by panel
  // (k_diag_factor + k_panel_trsm + k_trail_syrk, no grid barriers); the cooperative kernel's
  // 512-column outer panels keep the trailing updates of very large fronts
  // denser.
  bool panelFits(const Plan::Level& L) const {
    return panelMaxN > 0 && L.maxN <= panelMaxN && L.nf <= mfgpu::kMaxPanelFronts;
  }

  // Kernels that can factor level L (autotuning candidates).
  std::vector<int> levelCandidates(const Plan::Level& L) const {
    std::vector<int> c;
    if (L.nf <= 0) return c;
    if (mfgpu::small_front_fits(L.maxN, (int)esz)) c.push_back(LK_FUSED);
    if (mfgpu::coop_fits((int)L.nf) && !(stepped && !mixed)) {
      c.push_back(LK_COOP);
      if (L.nf <= mfgpu::kMaxPanelFronts) c.push_back(LK_PANEL);
      if (mixed && L.nf <= mfgpu::tc_max_fronts() && L.maxN >= 1024) c.push_back(LK_TC);
    }
    if (c.empty()) c.push_back(ruleKernel(L));
    return c;
  }

  // Panel-pack bytes a tensor-core run of level L needs (outer panels only when
  // the level was planned without sub-panels).
  size_t levelPackBytes(const Plan& P, const Plan::Level& L) const {
    std::vector<int> nn, NN;
    for (int64_t i = L.f0; i < L.f0 + L.nf; i++) {
      nn.push_back(S->fronts[realId(P, i)].n);
      NN.push_back(S->fronts[realId(P, i)].N);
    }
    size_t b = 0;
    const int W = mfgpu::tc_outer(), w = L.coopOuter > 0 ? L.coopOuter : W;
    for (int K = 0; K < L.maxn; K += w)
      for (int ww : {w, W})
        if (K % ww == 0)
          b = std::max(b, mfgpu::tc_pack_bytes((int)L.nf, mfgpu::tc_pack_cap(nn, NN, K, ww)));
    return b;
  }

  void dropGraphs(bool factor, bool sweep) {
    if (factor && fullGraph) {
      cudaGraphExecDestroy(fullGraph);
      fullGraph = nullptr;
    }
    if (sweep) {
      for (auto& kv : sweepGraphs)
        if (kv.second) cudaGraphExecDestroy(kv.second);
      sweepGraphs.clear();
      sweepSeen.clear();
    }
  }

  // The work fn enqueues on the stream, captured as an executable graph; null
  // (and graphs off for this handle) when the runtime refuses the capture.
  template <class Fn>
  cudaGraphExec_t capture(Fn&& fn) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
      cudaGetLastError();
      graphs = false;
      return nullptr;
    }
    bool ok = true;
    try {
      fn();
    } catch (const CudaError&) {
      ok = false;
    }
    if (cudaStreamEndCapture(stream, &g) != cudaSuccess || !ok || !g ||
        cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
      ex = nullptr;
      graphs = false;
    }
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();   // a refused capture leaves its error behind
    return ex;
  }

  // Launch the graph of (a, b, nc), capturing it on the second call with that
  // key; otherwise run fn directly.
  template <class Fn>
  void sweepGraph(const void* a, const void* b, int nc, Fn&& fn) {
    if (!graphs || prof.verbose) return fn();
    const auto key = std::make_tuple(a, b, nc);
    auto it = sweepGraphs.find(key);
    if (it == sweepGraphs.end() && ++sweepSeen[key] >= 2) {
      cudaGraphExec_t ex = capture(fn);
      if (ex) it = sweepGraphs.emplace(key, ex).first;
    }
    if (it == sweepGraphs.end()) return fn();
    ck(cudaGraphLaunch(it->second, stream), "launch sweep graph");
  }

  void ensurePack(size_t bytes) {
    if (bytes <= tcPackCap) return;
    dropGraphs(true, false);   // the captured factorization reads the old pack
    ck(cudaStreamSynchronize(stream), "sync before growing the panel pack");
    cudaFree(d_tcpack);
    d_tcpack = nullptr;
    tcPackCap = 0;
    d_tcpack = dalloc<unsigned char>(bytes, "alloc tensor-core panel pack");
    tcPackCap = bytes;
  }

  // Partial factorization of the fronts of level ell with kernel `kind`.
  template <class T>
  void runLevelKernel(const Plan& P, const Plan::Level& L, int ell, int kind) {
    const Schedule& s = *S;
    T* F = (T*)d_F;
    double fl = 0;
    if (prof.on && kind != LK_STEPPED)
      for (int64_t i = L.f0; i < L.f0 + L.nf; i++) fl += s.front_flops(s.fronts[realId(P, i)]);
    if (kind == LK_FUSED) {
      prof.flops[MFGPU_KC_FRONT] += fl;
      prof.begin(MFGPU_KC_FRONT, stream);
      mfgpu::launch_front_small<T>(P.d_ids + L.f0, (int)L.nf, L.maxN, d_fr, F, d_err, stream);
      ck(cudaGetLastError(), "launch fused front factorization (k_front_small)");
      prof.end(stream);
    } else if (kind == LK_TC) {
      if (sizeof(T) != sizeof(float)) throw CudaError("tensor-core levels are mixed only", MFGPU_ERR_ARG);
      runTensorLevel(P, L, fl, ell);
    } else if (kind == LK_COOP) {
      prof.flops[MFGPU_KC_COOP] += fl;
      prof.begin(MFGPU_KC_COOP, stream);
      ck(mfgpu::launch_level_coop<T>(P.d_ids + L.f0, (int)L.nf, L.maxn, d_fr, F, d_err,
                                     (T*)d_slots, P.d_cpref + L.cpref0, d_gbar, stream, 0, -1, 0,
                                     1, L.coopItems, L.coopOuter),
         "launch cooperative level factorization (k_level_coop)");
      prof.end(stream);
    } else if (kind == LK_STEPPED) {
      if (sizeof(T) != sizeof(double))
        throw CudaError("no single-precision path for this level", MFGPU_ERR_ARG);
      runStepped(P, L);
    } else if (kind == LK_LU) {
      if (sizeof(T) != sizeof(double)) throw CudaError("LU fronts are FP64 only", MFGPU_ERR_ARG);
      runLU(P, L);
    } else if (kind == LK_PANEL) {
      prof.flops[MFGPU_KC_COOP] += fl;
      runPanel<T>(P, L);
    }
  }

  // Panel by panel (kernels_panel.cu): per W-column panel the barrier-free
  // panel factorization, then the trailing update of every front of the level.
  template <class T>
  void runPanel(const Plan& P, const Plan::Level& L) {
    const int W = mfgpu::panel_width((int)sizeof(T));
    for (int k = 0; k < L.maxn; k += W) {
      prof.begin(MFGPU_KC_COOP, stream);
      ck(mfgpu::launch_subpanel<T>(P.d_ids + L.f0, (int)L.nf, d_fr, (T*)d_F, k, W, (T*)d_pslot,
                                   d_err, stream),
         "launch panel factorization (k_diag_factor, k_panel_trsm)");
      ck(mfgpu::launch_trail_syrk<T>(P.d_ids + L.f0, (int)L.nf, d_fr, (T*)d_F, k, W, stream),
         "launch panel trailing update (k_trail_syrk)");
      prof.end(stream);
    }
  }

  // Pivoted LU of a level's fronts (nonsymmetric problems): per 32-column
  // step the panel, the row swaps and block-row solve, the trailing update
  // (kernels_lu.cu).  Flops: the LU form of a partial factorization,
  // 2n^3/3 + 2n^2 m + 2n m^2 per front, under the three profiling classes.
  void runLU(const Plan& P, const Plan::Level& L) {
    const Schedule& s = *S;
    double* F = (double*)d_F;
    const int* fl = P.d_ids + L.f0;
    for (int k = 0; k < L.maxn; k += mfgpu::kPanel) {
      if (prof.on) {
        for (int64_t i = L.f0; i < L.f0 + L.nf; i++) {
          const mfgpu::Front& f = s.fronts[realId(P, i)];
          if (k >= f.n) continue;
          const double kb = std::min(mfgpu::kPanel, f.n - k), M = f.N - k - kb;
          prof.flops[MFGPU_KC_POTRF] += kb * kb * kb / 3.0 + M * kb * kb;
          prof.flops[MFGPU_KC_TRSM] += M * kb * kb;
          prof.flops[MFGPU_KC_SYRK] += 2.0 * M * M * kb;
        }
      }
      const int cls[3] = {MFGPU_KC_POTRF, MFGPU_KC_TRSM, MFGPU_KC_SYRK};
      const char* what[3] = {"launch LU panel (k_lu_panel)", "launch LU swaps + block row (k_lu_swap_trsm)",
                             "launch LU trailing update (k_lu_gemm)"};
      for (int ph = 0; ph < 3; ph++) {
        prof.begin(cls[ph], stream);
        mfgpu::launch_lu_step(fl, (int)L.nf, L.maxN, d_fr, F, d_ipiv, k, d_err, stream, ph);
        ck(cudaGetLastError(), what[ph]);
        prof.end(stream);
      }
    }
  }

  // Run a factorization plan: per level, separator base assembly, front
  // assembly, partial Cholesky, separator accumulation (src/DE/mf2d.cpp:449-753).
  template <class T>
  void runPlanT(const Plan& P) {
    const Schedule& s = *S;
    size_t pack = P.tcPackBytes;   // tuned tensor-core levels may need more than the rules
    if (&P == &full)
      for (int ell = 0; ell < s.levels && ell < (int)tuned.size(); ell++)
        if (tuned[ell] == LK_TC) pack = std::max(pack, levelPackBytes(P, P.lv[ell]));
    ensurePack(pack);
    // the full factorization's schedule as one graph, from its second run on
    if (&P == &full && graphs && !prof.on && fullRuns++ > 0) {
      if (!fullGraph) fullGraph = capture([&] { enqueuePlanT<T>(P); });
      if (fullGraph) {
        ck(cudaGraphLaunch(fullGraph, stream), "launch factorization graph");
        return;
      }
    }
    enqueuePlanT<T>(P);
  }

  template <class T>
  void enqueuePlanT(const Plan& P) {
    const Schedule& s = *S;
    clearErr();
    for (int ell = s.levels - 1; ell >= 0; ell--) {
      const Plan::Level& L = P.lv[ell];
      prof.level = ell;
      runGroup<T>(P, L.sbase, groupBytes(P, L.sbase));
      runGroup<T>(P, L.ftask, groupBytes(P, L.ftask));
      if (L.subs.empty()) {
        runLevelKernel<T>(P, L, ell, levelKernel(P, L, ell));
      } else {
        for (const Plan::Level::Sub& u : L.subs) {
          Plan::Level Ls = L;
          Ls.f0 = u.f0;
          Ls.nf = u.nf;
          Ls.maxN = u.maxN;
          Ls.maxn = u.maxn;
          Ls.cpref0 = u.cpref0;
          Ls.coopItems = u.coopItems;
          Ls.coopOuter = u.coopOuter;
          runLevelKernel<T>(P, Ls, ell, u.kind);
        }
      }
      finishLevel<T>(P, L, ell);
    }
    ck(cudaGetLastError(), "factor launch");
  }

  // After a level's partial factorization: the cooperative sweeps' block
  // inverses, then the separator accumulation.
  template <class T>
  void finishLevel(const Plan& P, const Plan::Level& L, int ell) {
    if (L.nf > 0 && coopSweep(ell)) {
      mfgpu::launch_diag_inv<T>(P.d_ids + L.f0, (int)L.nf, L.maxn, d_fr, (T*)d_F, (T*)d_Dinv,
                                d_dinv_off, stream);
      ck(cudaGetLastError(), "launch diagonal-block inverses (k_diag_inv)");
    }
    runGroup<T>(P, L.sadd0, groupBytes(P, L.sadd0));
    runGroup<T>(P, L.sadd1, groupBytes(P, L.sadd1));
  }

  // Full factorization that also picks each level's kernel by timing: per
  // level, every candidate runs `reps` times on freshly assembled fronts (the
  // assembly rewrites every front element, as localized updates rely on) and
  // the fastest becomes the level's kernel for later full factorizations; the
  // level is then assembled and factored once more with it.
  template <class T>
  void autotuneT(int reps, int* choices) {
    const Schedule& s = *S;
    const Plan& P = full;
    tuned.assign(s.levels, LK_NONE);
    size_t pack = P.tcPackBytes;
    for (int ell = 0; ell < s.levels; ell++)
      for (int c : levelCandidates(P.lv[ell]))
        if (c == LK_TC) pack = std::max(pack, levelPackBytes(P, P.lv[ell]));
    ensurePack(pack);
    if (mixed) {
      mfgpu::launch_diag_scale(d_rp, d_ci, d_val, n, d_scale, d_iscale, stream);
      ck(cudaGetLastError(), "launch diagonal scaling");
    }
    clearErr();
    const bool prof_on = prof.on;
    prof.on = false;
    for (int ell = s.levels - 1; ell >= 0; ell--) {
      const Plan::Level& L = P.lv[ell];
      runGroup<T>(P, L.sbase, groupBytes(P, L.sbase));
      const std::vector<int> cand = levelCandidates(L);
      if (cand.size() > 1) {
        float best = 0;
        for (int c : cand) {
          float t = 0;
          for (int r = 0; r < std::max(1, reps); r++) {
            runGroup<T>(P, L.ftask, groupBytes(P, L.ftask));
            ck(cudaEventRecord(ev0, stream), "event");
            runLevelKernel<T>(P, L, ell, c);
            ck(cudaEventRecord(ev1, stream), "event");
            ck(cudaEventSynchronize(ev1), "autotune sync");
            float ms = 0;
            ck(cudaEventElapsedTime(&ms, ev0, ev1), "elapsed");
            t = r == 0 ? ms : std::min(t, ms);
          }
          if (tuned[ell] == LK_NONE || t < best) {
            tuned[ell] = c;
            best = t;
          }
        }
      }
      runGroup<T>(P, L.ftask, groupBytes(P, L.ftask));
      runLevelKernel<T>(P, L, ell, levelKernel(P, L, ell));
      finishLevel<T>(P, L, ell);
    }
    prof.on = prof_on;
    ck(cudaGetLastError(), "factor launch");
    if (choices)
      for (int ell = 0; ell < s.levels; ell++) choices[ell] = levelKernel(P, P.lv[ell], ell);
  }

  // One CTA per front (k_front_small) when the level has enough fronts to fill
  // the GPU and each front's staged panel fits in shared memory; otherwise the
  // cooperative kernel spreads every front of the level over all SMs (a
  // localized update often leaves one or two fronts per level).
  bool useFused(int nf, int maxN) const {
    return mfgpu::small_front_fits(maxN, (int)esz) && (nf >= fusedMinFronts || maxN <= 64);
  }

  // Mixed path: levels of large fronts run the cooperative kernel one outer
  // panel at a time (diagonal blocks, panel solves and in-panel updates) and
  // the trailing update of each panel on the tensor cores.
  // A level also goes to the tensor cores with fronts of a quarter of tcMinN
  // when it has at least one front per SM (enough tiles to fill the GPU; 3D
  // 127^3 level 3: 512 fronts, N <= 1981); levels with a few such fronts (the
  // top of a 2D tree) stay on the cooperative kernel, which is faster there.
  bool tcLevel(const Plan::Level& L) const {
    if (tcMinN <= 0 || L.nf > mfgpu::tc_max_fronts()) return false;
    return L.maxN >= tcMinN || (L.nf >= 148 && L.maxN >= tcMinN / 4);
  }

  // Tensor-core level (mixed path).  Per 512-column outer panel [K, K + 512):
  // the cooperative kernel factors it one sub-panel [Ks, Ks + w) at a time
  // (w = L.coopOuter, 32-column steps inside), and after each sub-panel the
  // tensor cores update the outer panel's remaining columns [Ks + w, K + 512)
  // of all rows below; then the tensor cores apply the whole outer panel to
  // the trailing matrix.  With w = 512 (no sub-panels) only the trailing
  // update remains.  Profile attribution: the tensor-core updates'
  // algorithmic flops go to MFGPU_KC_TC, the rest of the level's flops
  // (diagonal blocks, panel solves, in-sub-panel updates) to MFGPU_KC_COOP.
  void runTensorLevel(const Plan& P, const Plan::Level& L, double level_flops, int ell) {
    const Schedule& s = *S;
    const int split = tcSplit3Levels >= 0 && ell >= tcSplit3Levels ? tcSplitLow : tcSplit;
    std::vector<int> nn(L.nf), NN(L.nf);
    for (int64_t i = 0; i < L.nf; i++) {
      nn[i] = s.fronts[realId(P, L.f0 + i)].n;
      NN[i] = s.fronts[realId(P, L.f0 + i)].N;
    }
    const int W = mfgpu::tc_outer(), w = L.coopOuter > 0 ? L.coopOuter : W;
    int phase0 = 0;
    double tc_fl = 0;
    // C(k1:N, k1:cmax) -= P P^T for the panel [K0, K0 + pw), cmax = min(cend, n) (cend < 0: N)
    auto update = [&](int K0, int pw, int cend) {
      const int64_t nt = mfgpu::tc_tiles(nn, NN, K0, pw, cend);
      if (nt == 0) return;
      if (prof.on)
        for (int64_t i = 0; i < L.nf; i++)
          if (K0 < nn[i]) {
            const double k1 = std::min(K0 + pw, nn[i]);
            const double c = cend < 0 ? NN[i] : std::min(cend, nn[i]);
            if (c <= k1) continue;
            // lower-triangle entries of rows [k1, N) x columns [k1, c), one
            // multiply-add per entry and panel column
            const double r = NN[i] - k1, cw = c - k1;
            tc_fl += 2.0 * cw * (r - 0.5 * cw) * (k1 - K0);
          }
      const int cap = mfgpu::tc_pack_cap(nn, NN, K0, pw);
      if (mfgpu::tc_pack_bytes((int)L.nf, cap) > tcPackCap)
        throw CudaError("tensor-core panel pack larger than planned", MFGPU_ERR_STATE);
      prof.begin(MFGPU_KC_TC, stream);
      ck(mfgpu::launch_tc_pack(P.d_ids + L.f0, (int)L.nf, cap, d_fr, (const float*)d_F, K0, pw,
                               split, d_tcpack, stream),
         "launch tensor-core panel pack (k_tc_pack)");
      ck(mfgpu::launch_trail_tc(P.d_ids + L.f0, (int)L.nf, nt, d_fr, (float*)d_F, K0, pw, cend,
                                split, cap, d_tcpack, d_err, stream),
         "launch tensor-core update (k_trail_tc)");
      prof.end(stream);
    };
    for (int K = 0; K < L.maxn; K += W) {
      for (int Ks = K; Ks < K + W && Ks < L.maxn; Ks += w) {
        prof.begin(MFGPU_KC_COOP, stream);
        if (subpanel && w == mfgpu::panel_width(sizeof(float)) && L.nf <= mfgpu::kMaxPanelFronts) {
          ck(mfgpu::launch_subpanel<float>(P.d_ids + L.f0, (int)L.nf, d_fr, (float*)d_F, Ks, w,
                                           (float*)d_pslot, d_err, stream),
             "launch sub-panel factorization (k_diag_factor, k_panel_trsm)");
        } else {
          ck(mfgpu::launch_level_coop<float>(P.d_ids + L.f0, (int)L.nf, L.maxn, d_fr, (float*)d_F,
                                             d_err, (float*)d_slots, P.d_cpref + L.cpref0, d_gbar,
                                             stream, Ks, Ks + w, phase0, 0, L.coopItems, w),
             "launch cooperative panel factorization (k_level_coop)");
        }
        prof.end(stream);
        phase0 += mfgpu::coop_phases(Ks, L.maxn, w);
        if (Ks + w < K + W) update(Ks, w, K + W);   // the outer panel's remaining columns
      }
      update(K, W, -1);   // the trailing matrix
    }
    prof.flops[MFGPU_KC_TC] += tc_fl;
    prof.flops[MFGPU_KC_COOP] += std::max(0.0, level_flops - tc_fl);
  }

  // FP64 per-step launches (MFGPU_STEPPED=1, or levels no cooperative launch takes).
  void runStepped(const Plan& P, const Plan::Level& L) {
    const Schedule& s = *S;
    double* F = (double*)d_F;
    const int* fl = P.d_ids + L.f0;
    for (int k = 0; k < L.maxn; k += mfgpu::kPanel) {
      if (prof.on) {
        for (int64_t i = L.f0; i < L.f0 + L.nf; i++) {
          const mfgpu::Front& f = s.fronts[realId(P, i)];
          if (k >= f.n) continue;
          double kb = std::min(mfgpu::kPanel, f.n - k), M = f.N - k - kb;
          prof.flops[MFGPU_KC_POTRF] += kb * kb * kb / 3.0;
          prof.flops[MFGPU_KC_TRSM] += M * kb * kb;
          prof.flops[MFGPU_KC_SYRK] += M * M * kb;
        }
      }
      prof.begin(MFGPU_KC_POTRF, stream);
      mfgpu::launch_potrf(fl, (int)L.nf, d_fr, F, k, d_err, stream);
      ck(cudaGetLastError(), "launch panel Cholesky (k_potrf)");
      prof.end(stream);
      prof.begin(MFGPU_KC_TRSM, stream);
      mfgpu::launch_trsm(fl, (int)L.nf, d_fr, F, k, L.maxN, stream);
      ck(cudaGetLastError(), "launch panel solve (k_trsm)");
      prof.end(stream);
      prof.begin(MFGPU_KC_SYRK, stream);
      mfgpu::launch_syrk(fl, (int)L.nf, d_fr, F, k, L.maxN, stream);
      ck(cudaGetLastError(), "launch trailing update (k_syrk)");
      prof.end(stream);
    }
  }

  void runPlan(const Plan& P) {
    if (mixed) runPlanT<float>(P);
    else runPlanT<double>(P);
  }

  // Replace the matrix values (same pattern) and refactor a plan.  The mixed
  // path's diagonal scaling is recomputed only with a full factorization and
  // kept through localized updates, so fronts that an update leaves alone stay
  // consistent with the ones it recomputes.
  void factorWith(const double* val, bool device, const Plan& P, bool full) {
    if (val)
      ck(cudaMemcpyAsync(d_val, val, nnz * sizeof(double),
                         device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, stream),
         "upload values");
    if (mixed && full) {
      mfgpu::launch_diag_scale(d_rp, d_ci, d_val, n, d_scale, d_iscale, stream);
      ck(cudaGetLastError(), "launch diagonal scaling");
    }
    runPlan(P);
  }

  // Reset the error word before a call's launches (a memset, so it can be
  // captured in a graph); its poll-limit field is written only by setLimit.
  void clearErr() {
    ck(cudaMemsetAsync(d_err, 0, offsetof(DevError, limit), stream), "clear error word");
  }
  void setLimit(unsigned polls) {
    waitLimit = polls;
    ck(cudaMemcpyAsync(&d_err->limit, &waitLimit, sizeof(unsigned), cudaMemcpyHostToDevice, stream),
       "set wait limit");
    ck(cudaStreamSynchronize(stream), "set wait limit");
  }

  void checkDevError() {
    DevError e;
    ck(cudaMemcpyAsync(&e, d_err, sizeof(e), cudaMemcpyDeviceToHost, stream), "read error word");
    ck(cudaStreamSynchronize(stream), "factor");
    if (e.code == 2 || e.code == 3) {
      throw CudaError(e.code == 2 ? "a tensor-core pipeline wait gave up (k_trail_tc)"
                                  : "a cooperative kernel's grid barrier gave up",
                      MFGPU_ERR_TIMEOUT);
    }
    if (e.code == 4) {
      const mfgpu::Front& f = S->fronts[e.front % (int)S->fronts.size()];
      char buf[256];
      snprintf(buf, sizeof buf,
               "zero pivot column in front %d (level %d, box %d) at pivot column %d: the front's "
               "pivot block is singular",
               e.front, f.level, f.box, e.col);
      throw CudaError(buf, MFGPU_ERR_PIVOT);
    }
    if (e.code == 1) {
      const mfgpu::Front& f = S->fronts[e.front % (int)S->fronts.size()];
      char buf[256];
      snprintf(buf, sizeof buf,
               "non-positive pivot in front %d (level %d, box %d) at pivot column %d: the matrix "
               "is not symmetric positive definite",
               e.front, f.level, f.box, e.col);
      throw CudaError(buf, MFGPU_ERR_PIVOT);
    }
  }

  // ---- solve / apply buffers ----
  template <class P>
  void growBuf(P*& p, size_t& cap, size_t need, const char* what) {
    if (need <= cap) return;
    dropGraphs(false, true);   // captured sweeps read the old buffers
    cudaFree(p);
    p = nullptr;
    p = dalloc<P>(need, what);
    cap = need;
  }

  void ensureWork(int nrhs) {
    growBuf(d_Wd, capW, (size_t)woffTotal * nrhs * esz / sizeof(double) + 1, "alloc solve workspace");
    growBuf(d_X, capX, (size_t)n * nrhs, "alloc rhs buffer");
    growBuf(d_Td, capT, (size_t)n * nrhs * esz / sizeof(double) + 1, "alloc apply buffer");
    if (mixed) {
      const size_t v = (size_t)n * nrhs;
      growBuf(d_B, capB, v, "alloc refinement buffer");
      growBuf(d_R, capR, v, "alloc refinement buffer");
      growBuf(d_P, capP, v, "alloc refinement buffer");
      growBuf(d_Q, capQ, v, "alloc refinement buffer");
      growBuf(d_Z, capZ, v, "alloc refinement buffer");
      growBuf(d_x32, cap32, v, "alloc refinement buffer");
      growBuf(d_dotp, capDot, (size_t)nchunks * nrhs, "alloc dot scratch");
    }
  }

  // MFGPU_VERBOSE: per-level marks inside the solve (class SOLVE, level tag).
  void vmark(bool begin, int level) {
    if (!prof.verbose) return;
    if (begin) {
      prof.level = level;
      prof.begin(MFGPU_KC_SOLVE, stream);
    } else {
      prof.end(stream);
    }
  }

  // Forward / backward sweeps of the factorization in precision T, in place on
  // X (n x nrhs, ld ldx, nrhs <= 16) with per-front workspace W
  // (src/DE/mf2d.cpp:976-1054).
  bool coopSweep(int ell) const {
    return solveCoopMinN > 0 && lvMaxN[ell] >= solveCoopMinN &&
           S->lv[ell].nbox <= mfgpu::solve_coop_max_fronts();
  }

  template <class T>
  void sweepLevel(bool forward, int ell, T* X, int64_t ldx, int nrhs, T* W) {
    const Schedule& s = *S;
    const T* F = (const T*)d_F;
    const int* fl = d_all + s.lv[ell].front0;
    const int nf = s.lv[ell].nbox;
    if (lu) {
      if (sizeof(T) != sizeof(double)) throw CudaError("LU fronts are FP64 only", MFGPU_ERR_ARG);
      mfgpu::launch_lu_solve(forward, fl, nf, lvMaxN[ell], d_fr, (const double*)F, d_ipiv, d_dofs,
                             (double*)X, ldx, nrhs, (double*)W, d_woff, stream);
      ck(cudaGetLastError(), forward ? "launch LU forward sweep (k_lu_solve_fwd)"
                                     : "launch LU backward sweep (k_lu_solve_bwd)");
    } else if (coopSweep(ell)) {
      const FlowLevel& q = flow[ell];
      ck(mfgpu::launch_solve_flow<T>(forward, fl, d_fr, F, d_dofs, X, ldx, nrhs, W, d_woff,
                                     (const T*)d_Dinv, d_dinv_off,
                                     d_flow + (forward ? q.fwd : q.bwd), forward ? q.nfwd : q.nbwd,
                                     d_flow + q.flagoff, d_flags, q.nflags, d_err, stream),
         forward ? "launch cooperative forward sweep (k_solve_flow_fwd)"
                 : "launch cooperative backward sweep (k_solve_flow_bwd)");
    } else if (forward) {
      mfgpu::launch_solve_fwd<T>(fl, nf, lvMaxN[ell], d_fr, F, d_dofs, X, ldx, nrhs, W, d_woff,
                                 stream);
      ck(cudaGetLastError(), "launch forward sweep (k_solve_fwd)");
    } else {
      mfgpu::launch_solve_bwd<T>(fl, nf, lvMaxN[ell], d_fr, F, d_dofs, X, ldx, nrhs, W, d_woff,
                                 stream);
      ck(cudaGetLastError(), "launch backward sweep (k_solve_bwd)");
    }
  }

  // Forward / backward sweeps of the factorization in precision T, in place on
  // X (n x nrhs, ld ldx, nrhs <= 16) with per-front workspace W
  // (src/DE/mf2d.cpp:976-1054).
  template <class T>
  void sweeps(T* X, int64_t ldx, int nrhs, T* W) {
    const Schedule& s = *S;
    const T* F = (const T*)d_F;
    for (int ell = s.levels - 1; ell >= 1; ell--) {
      const int s0 = s.lv[ell].sep0;
      vmark(true, ell);
      sweepLevel<T>(true, ell, X, ldx, nrhs, W);
      vmark(false, ell);
      mfgpu::launch_sep_gather<T>(d_all + s.fronts.size() + s0, s.lv[ell].nsep, d_sp, d_dofs, X, ldx,
                                  nrhs, W, d_woff, d_fr, stream);
      ck(cudaGetLastError(), "launch separator gather (k_sep_gather)");
    }
    vmark(true, 0);
    if (lu || coopSweep(0) || s.lv[0].nbox > 1) {   // several roots (a batch), LU: generic sweeps
      sweepLevel<T>(true, 0, X, ldx, nrhs, W);
      sweepLevel<T>(false, 0, X, ldx, nrhs, W);
    } else {
      mfgpu::launch_root_solve<T>(0, s.fronts[0].N, d_fr, F, d_dofs, X, ldx, nrhs, W, d_woff, stream);
      ck(cudaGetLastError(), "launch root solve (k_root_solve)");
    }
    vmark(false, 0);
    for (int ell = 1; ell < s.levels; ell++) {
      vmark(true, 100 + ell);
      sweepLevel<T>(false, ell, X, ldx, nrhs, W);
      vmark(false, 100 + ell);
    }
  }

  // Factored-operator application in precision T (src/DE/mf2d.cpp:904-974).
  template <class T>
  void applySweeps(T* X, int64_t ldx, int nrhs, T* W, T* Tb) {
    const Schedule& s = *S;
    const T* F = (const T*)d_F;
    auto up = [&](int ell) {
      if (lu) {
        mfgpu::launch_lu_apply_up(d_all + s.lv[ell].front0, s.lv[ell].nbox, d_fr, (const double*)F,
                                  d_ipiv, d_dofs, (double*)X, ldx, nrhs, (double*)W, d_woff,
                                  (double*)Tb, stream);
        ck(cudaGetLastError(), "launch LU apply up (k_lu_apply_up)");
      } else {
        mfgpu::launch_apply_up<T>(d_all + s.lv[ell].front0, s.lv[ell].nbox, d_fr, F, d_dofs, X, ldx,
                                  nrhs, W, d_woff, Tb, stream);
        ck(cudaGetLastError(), "launch apply up (k_apply_up)");
      }
    };
    for (int ell = s.levels - 1; ell >= 1; ell--) up(ell);
    if (lu) {
      up(0);
    } else if (s.lv[0].nbox > 1) {   // several roots (a batch)
      mfgpu::launch_apply_up<T>(d_all, s.lv[0].nbox, d_fr, F, d_dofs, X, ldx, nrhs, W, d_woff, Tb,
                                stream);
      ck(cudaGetLastError(), "launch apply up (k_apply_up)");
    } else {
      mfgpu::launch_root_apply<T>(0, d_fr, F, d_dofs, X, ldx, nrhs, W, d_woff, stream);
      ck(cudaGetLastError(), "launch root apply (k_root_apply)");
    }
    for (int ell = 1; ell < s.levels; ell++) {
      mfgpu::launch_apply_down<T>(d_all + s.lv[ell].front0, s.lv[ell].nbox, d_fr, F, d_dofs, ldx,
                                  nrhs, W, d_woff, Tb, stream);
      ck(cudaGetLastError(), "launch apply down (k_apply_down)");
      mfgpu::launch_sep_gather<T>(d_all + s.fronts.size() + s.lv[ell].sep0, s.lv[ell].nsep, d_sp,
                                  d_dofs, X, ldx, nrhs, W, d_woff, d_fr, stream);
      ck(cudaGetLastError(), "launch separator gather (k_sep_gather)");
    }
  }

  // z = M^{-1} r with the scaled FP32 factorization: z = s .* (S^{-1} (s .* r)).
  void precond(const double* r, double* z, int nc) {
    sweepGraph(r, z, nc, [&] {
      mfgpu::launch_scale_to<float>(r, n, d_x32, n, d_scale, n, nc, stream);
      sweeps<float>(d_x32, n, nc, (float*)d_Wd);
      mfgpu::launch_scale_from<float>(d_x32, n, z, n, d_scale, n, nc, stream);
    });
  }

  void dots(const double* x, const double* y, int nc, double* out) {
    mfgpu::launch_dot(x, n, y, n, nc, d_chunkrow, nchunks, d_segchunk, nseg, d_dotp, out, stream);
  }

  // Mixed precision: conjugate gradients on A x = b in FP64 (residuals from the
  // FP64 CSR matrix), preconditioned by the FP32 factorization, until
  // ||b - A x|| <= tol ||b|| for every column.  XB holds b on entry, x on exit
  // (n x nc, ld n).
  void pcg(double* XB, int nc) {
    const double tol = opt.refine_tol > 0 ? opt.refine_tol : 1e-10;
    const int maxit = opt.refine_maxit > 0 ? opt.refine_maxit : 50;
    const size_t vb = (size_t)n * nc * sizeof(double);
    const int G = nseg * nc;            // (segment, column) pairs
    double* rzA = d_sc;                 // rz_a | rz_b | pq | rr | bb, nseg * 16 each
    double* rzB = d_sc + 16 * nseg;
    double* pq = d_sc + 32 * nseg;
    double* rr = d_sc + 48 * nseg;
    double* bb = d_sc + 64 * nseg;
    ck(cudaMemcpyAsync(d_B, XB, vb, cudaMemcpyDeviceToDevice, stream), "copy rhs");
    dots(d_B, d_B, nc, bb);
    precond(d_B, XB, nc);   // x0 = M^{-1} b
    mfgpu::launch_residual(d_rp, d_ci, d_val, n, d_B, n, XB, n, d_R, n, nc, stream);
    std::vector<double> hb(G), hr(G);
    std::vector<int> act(G);
    ck(cudaMemcpyAsync(hb.data(), bb, G * sizeof(double), cudaMemcpyDeviceToHost, stream),
       "read norms");
    int it = 0, restarts = 0;
    bool first = true;
    double worst = 0;
    // relative residual of every (segment, column); returns how many miss tol
    auto check = [&]() {
      dots(d_R, d_R, nc, rr);
      ck(cudaMemcpyAsync(hr.data(), rr, G * sizeof(double), cudaMemcpyDeviceToHost, stream),
         "read norms");
      ck(cudaStreamSynchronize(stream), "refinement");
      int nact = 0;
      worst = 0;
      for (int g = 0; g < G; g++) {
        const double rel = hb[g] > 0 ? std::sqrt(hr[g] / hb[g]) : std::sqrt(hr[g]);
        worst = std::max(worst, rel);
        act[g] = rel > tol;
        nact += act[g];
      }
      return nact;
    };
    while (true) {
      if (check() == 0) {
        // confirm with the true residual; restart from it if the recursive one drifted
        mfgpu::launch_residual(d_rp, d_ci, d_val, n, d_B, n, XB, n, d_R, n, nc, stream);
        if (check() == 0 || restarts >= 3) break;
        restarts++;
        first = true;
      }
      if (it >= maxit) break;
      ck(cudaMemcpyAsync(d_active, act.data(), G * sizeof(int), cudaMemcpyHostToDevice, stream),
         "flags");
      precond(d_R, d_Z, nc);
      dots(d_R, d_Z, nc, rzB);
      mfgpu::launch_pcg_p(d_P, d_Z, n, n, nc, rzB, rzA, d_active, first ? 1 : 0, d_segrow, nseg,
                          stream);
      mfgpu::launch_spmv(d_rp, d_ci, d_val, n, d_P, n, d_Q, n, nc, stream);
      dots(d_P, d_Q, nc, pq);
      mfgpu::launch_pcg_xr(XB, d_R, d_P, d_Q, n, n, nc, rzB, pq, d_active, d_segrow, nseg, stream);
      ck(cudaGetLastError(), "refinement launch");
      std::swap(rzA, rzB);   // rz of this iteration becomes the previous one
      first = false;
      it++;
    }
    stats.iterations = std::max(stats.iterations, it);
    stats.residual = std::max(stats.residual, worst);
    if (worst > tol) {
      char buf[160];
      snprintf(buf, sizeof buf,
               "refinement stopped after %d iterations at relative residual %.3e (target %.1e)", it,
               worst, tol);
      throw CudaError(buf, MFGPU_ERR_NOT_CONVERGED);
    }
  }

  // Solve in place on device data X (n x nrhs, ld = n), nrhs <= 16.
  void solveChunk(double* X, int nrhs) {
    if (mixed) pcg(X, nrhs);
    else sweepGraph(X, d_Wd, nrhs, [&] { sweeps<double>(X, n, nrhs, (double*)d_Wd); });
    ck(cudaGetLastError(), "solve launch");
  }

  // The FP64 sweeps with the per-front workspace at W (used by the
  // no-allocation entry point, which passes its static scratch).
  void solveChunkScratch(double* X, int64_t ldx, int nrhs, double* W) {
    sweeps<double>(X, ldx, nrhs, W);
    ck(cudaGetLastError(), "solve launch");
  }

  // b = (factored A) x in place on X (n x nrhs, ld n).  The mixed path applies
  // the scaled FP32 factorization: A ~ D^{1/2} L L^T D^{1/2}, D^{1/2} = 1/s.
  void applyChunk(double* X, int nrhs) {
    if (!mixed) {
      applySweeps<double>(X, n, nrhs, (double*)d_Wd, (double*)d_Td);
    } else {
      mfgpu::launch_scale_to<float>(X, n, d_x32, n, d_iscale, n, nrhs, stream);
      applySweeps<float>(d_x32, n, nrhs, (float*)d_Wd, (float*)d_Td);
      mfgpu::launch_scale_from<float>(d_x32, n, X, n, d_iscale, n, nrhs, stream);
    }
    ck(cudaGetLastError(), "apply launch");
  }
};

namespace {

int fail(mfgpu_handle* h, int status, const std::string& msg) {
  if (h) h->err = msg;
  return status;
}

template <class F>
int guarded(mfgpu_handle* h, F&& fn) {
  if (!h) return MFGPU_ERR_ARG;
  try {
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(h, MFGPU_ERR_CUDA, "cudaSetDevice failed");
    fn();
    h->err.clear();
    return MFGPU_OK;
  } catch (const CudaError& e) {
    return fail(h, e.status, e.what());
  } catch (const std::bad_alloc&) {
    return fail(h, MFGPU_ERR_OOM, "host allocation failed");
  } catch (const std::invalid_argument& e) {
    return fail(h, MFGPU_ERR_ARG, e.what());
  } catch (const std::exception& e) {
    return fail(h, MFGPU_ERR_CUDA, e.what());
  }
}

thread_local std::string g_create_error;
thread_local std::string g_sym_error;

}  // namespace

extern "C" {

void mfgpu_default_options(mfgpu_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->precision = MFGPU_FP64;
  o->device = 0;
  o->refine_tol = 1e-10;
  o->refine_maxit = 50;
}

const char* mfgpu_status_string(int s) {
  switch (s) {
    case MFGPU_OK: return "ok";
    case MFGPU_ERR_ARG: return "invalid argument";
    case MFGPU_ERR_DEPTH: return "recursion depth is 1 level";
    case MFGPU_ERR_LEAF: return "leaf box arithmetic failed";
    case MFGPU_ERR_OOM: return "out of device memory";
    case MFGPU_ERR_CUDA: return "CUDA error";
    case MFGPU_ERR_PIVOT: return "non-positive pivot (matrix not SPD)";
    case MFGPU_ERR_TIMEOUT: return "device wait timed out";
    case MFGPU_ERR_STATE: return "call out of order";
    case MFGPU_ERR_NOT_CONVERGED: return "refinement did not converge";
  }
  return "unknown status";
}

namespace {

// Schedule of one problem; the reference's constructor exceptions become
// status codes (src/DE/mf2d.cpp:38-43 recursion depth, :60-66 leaf math).
// Separator widths 2-3 (the reference fixture's wider stencils,
// test_include/DE/buildLaplacian.hpp:18-35) give nonsymmetric operators: their
// schedule carries full-storage task tables and the handle factors by pivoted
// LU.  Batches take width 1 only.
int makeSchedule(int dim, int nx, int ny, int nz, int width, int max_side,
                 std::unique_ptr<Schedule>& out, bool allow_wide = true) {
  if (width < 1 || width > 3 || (!allow_wide && width != 1)) {
    g_create_error = allow_wide ? "separator width must be 1, 2 or 3"
                                : "batch members must have separator width 1";
    return MFGPU_ERR_ARG;
  }
  try {
    out.reset(new Schedule(dim, nx, ny, nz, width, max_side, /*full_storage=*/width > 1));
  } catch (const std::invalid_argument& e) {
    g_create_error = e.what();
    return MFGPU_ERR_ARG;
  } catch (const std::runtime_error& e) {
    g_create_error = e.what();
    return std::string(e.what()).find("recursion depth") != std::string::npos ? MFGPU_ERR_DEPTH
                                                                                : MFGPU_ERR_LEAF;
  }
  return MFGPU_OK;
}

int createFrom(std::unique_ptr<Schedule> sched, int n, const int* row_ptr, const int* col_ind,
               const double* val, const mfgpu_options* opts, mfgpu_handle** out);

// The factorization reads the lower triangle only, so a matrix that is not
// symmetric would be factored as another one.  Returns why the CSR matrix is
// not symmetric (entries (i, j) and (j, i) both stored and equal to a
// relative 1e-12), or nullptr.  Rows need not be sorted.
const char* asymmetry(int n, const int* rp, const int* ci, const double* val,
                      std::string& where) {
  for (int i = 0; i < n; i++) {
    if (rp[i + 1] < rp[i]) return "row pointers decrease";
    for (int p = rp[i]; p < rp[i + 1]; p++) {
      const int j = ci[p];
      if (j < 0 || j >= n) return "column index out of range";
      if (j == i) continue;
      int q = rp[j];
      while (q < rp[j + 1] && ci[q] != i) q++;
      const bool ok = q < rp[j + 1] && std::fabs(val[p] - val[q]) <=
                                           1e-12 * std::max(std::fabs(val[p]), std::fabs(val[q]));
      if (!ok) {
        where = " (entries (" + std::to_string(i) + ", " + std::to_string(j) + ") and (" +
                std::to_string(j) + ", " + std::to_string(i) + "))";
        return "the matrix is not symmetric";
      }
    }
  }
  return nullptr;
}

}  // namespace

int mfgpu_create(int dim, int nx, int ny, int nz, int width, int max_side, int n,
                 const int* row_ptr, const int* col_ind, const double* val,
                 const mfgpu_options* opts, mfgpu_handle** out) {
  if (!out) return MFGPU_ERR_ARG;
  *out = nullptr;
  g_create_error.clear();
  if (!row_ptr || !col_ind || !val) {
    g_create_error = "null CSR pointer";
    return MFGPU_ERR_ARG;
  }
  std::unique_ptr<Schedule> sched;
  const int st = makeSchedule(dim, nx, ny, nz, width, max_side, sched);
  if (st != MFGPU_OK) return st;
  return createFrom(std::move(sched), n, row_ptr, col_ind, val, opts, out);
}

int mfgpu_batch_create(int count, const int* dim, const int* nx, const int* ny, const int* nz,
                       const int* width, const int* max_side, int n, const int* row_ptr,
                       const int* col_ind, const double* val, const mfgpu_options* opts,
                       mfgpu_handle** out) {
  if (!out) return MFGPU_ERR_ARG;
  *out = nullptr;
  g_create_error.clear();
  if (count <= 0 || !dim || !nx || !ny || !nz || !width || !max_side || !row_ptr || !col_ind ||
      !val) {
    g_create_error = "bad batch arguments";
    return MFGPU_ERR_ARG;
  }
  std::vector<Schedule> parts;
  parts.reserve(count);
  for (int p = 0; p < count; p++) {
    std::unique_ptr<Schedule> one;
    const int st = makeSchedule(dim[p], nx[p], ny[p], nz[p], width[p], max_side[p], one, false);
    if (st != MFGPU_OK) {
      g_create_error = "batch member " + std::to_string(p) + ": " + g_create_error;
      return st;
    }
    parts.push_back(std::move(*one));
  }
  std::unique_ptr<Schedule> sched;
  try {
    sched.reset(new Schedule(std::move(parts)));
  } catch (const std::exception& e) {
    g_create_error = e.what();
    return MFGPU_ERR_ARG;
  }
  return createFrom(std::move(sched), n, row_ptr, col_ind, val, opts, out);
}

int mfgpu_batch_info(const mfgpu_handle* h, int* count, int64_t* dof_offsets) {
  if (!h) return MFGPU_ERR_ARG;
  const Schedule& s = *h->S;
  const int c = s.forest() ? (int)s.parts.size() : 1;
  if (count) *count = c;
  if (dof_offsets) {
    if (s.forest())
      for (int p = 0; p <= c; p++) dof_offsets[p] = s.dof_base[p];
    else
      dof_offsets[0] = 0, dof_offsets[1] = s.ndof;
  }
  return MFGPU_OK;
}

namespace {

int createFrom(std::unique_ptr<Schedule> sched, int n, const int* row_ptr, const int* col_ind,
               const double* val, const mfgpu_options* opts, mfgpu_handle** out) {
  std::unique_ptr<mfgpu_handle> h(new (std::nothrow) mfgpu_handle());
  if (!h) return MFGPU_ERR_OOM;
  mfgpu_default_options(&h->opt);
  if (opts) h->opt = *opts;
  h->device = h->opt.device;
  if (h->opt.precision != MFGPU_FP64 && h->opt.precision != MFGPU_MIXED) {
    g_create_error = "unknown precision";
    return MFGPU_ERR_ARG;
  }
  h->S = std::move(sched);
  const Schedule& s = *h->S;
  if ((int64_t)n != s.ndof || row_ptr[0] != 0) {
    g_create_error = "matrix dimension does not match the grid";
    return MFGPU_ERR_ARG;
  }
  h->lu = s.full_storage;
  if (h->lu && h->opt.precision != MFGPU_FP64) {
    g_create_error = "separator widths 2-3 (nonsymmetric operators, pivoted LU) are FP64 only";
    return MFGPU_ERR_ARG;
  }
  std::string where;
  if (!h->lu)
    if (const char* why = asymmetry(n, row_ptr, col_ind, val, where)) {
      g_create_error = std::string(why) + where +
                       ": this library factors symmetric positive definite matrices with "
                       "separator width 1 (widths 2-3 are factored by pivoted LU)";
      return MFGPU_ERR_ARG;
    }
  h->n = n;
  h->nnz = row_ptr[n];
  if (const char* e = getenv("MFGPU_STEPPED")) h->stepped = e[0] == '1';
  if (const char* e = getenv("MFGPU_VERBOSE")) h->prof.verbose = e[0] == '1';
  if (const char* e = getenv("MFGPU_TC_MIN_N")) h->tcMinN = atoi(e);
  if (const char* e = getenv("MFGPU_SOLVE_COOP_MIN_N")) h->solveCoopMinN = atoi(e);
  if (const char* e = getenv("MFGPU_FUSED_MIN_FRONTS")) h->fusedMinFronts = atoi(e);
  auto splitOf = [](const char* e, int dflt) {
    const std::string v(e);
    return v == "1" || v == "tf32" ? 1 : v == "bf16" ? 2 : v == "3" ? 3 : dflt;
  };
  if (const char* e = getenv("MFGPU_TC_SPLIT")) h->tcSplit = splitOf(e, 3);
  if (const char* e = getenv("MFGPU_TC_LOW")) h->tcSplitLow = splitOf(e, 1);
  if (const char* e = getenv("MFGPU_TC_SPLIT3_LEVELS")) h->tcSplit3Levels = atoi(e);
  if (const char* e = getenv("MFGPU_TC_SUB")) h->tcSub = atoi(e);
  if (const char* e = getenv("MFGPU_GRAPHS")) h->graphs = e[0] != '0';
  if (const char* e = getenv("MFGPU_SUBPANEL")) h->subpanel = e[0] != '0';
  if (const char* e = getenv("MFGPU_PANEL_MAX_N")) h->panelMaxN = atoi(e);
  if (h->lu) h->solveCoopMinN = 0;   // LU fronts use the per-front sweeps
  h->h_rowptr.assign(row_ptr, row_ptr + n + 1);
  h->h_colind.assign(col_ind, col_ind + h->nnz);
  int st = guarded(h.get(), [&]() {
    mfgpu_handle& H = *h;
    ck(cudaStreamCreateWithFlags(&H.own, cudaStreamNonBlocking), "create stream");
    H.stream = H.own;
    ck(cudaEventCreate(&H.ev0), "event");
    ck(cudaEventCreate(&H.ev1), "event");
    H.mixed = H.opt.precision == MFGPU_MIXED;
    H.esz = H.mixed ? sizeof(float) : sizeof(double);
    H.d_F = dalloc<unsigned char>(s.front_elems * H.esz, "alloc front arena");
    H.d_Sep = dalloc<unsigned char>(s.sep_elems * H.esz, "alloc separator arena");
    if (H.mixed) {
      std::vector<int64_t> segrow = s.forest() ? s.dof_base : std::vector<int64_t>{0, s.ndof};
      H.nseg = (int)segrow.size() - 1;
      std::vector<int> chunkrow, segchunk, segrow32(segrow.begin(), segrow.end());
      mfgpu::dot_plan(segrow, chunkrow, segchunk);
      H.nchunks = (int)chunkrow.size() - 1;
      H.d_scale = dalloc<double>(n, "alloc scaling");
      H.d_iscale = dalloc<double>(n, "alloc scaling");
      H.d_sc = dalloc<double>(80 * (size_t)H.nseg, "alloc refinement scalars");
      H.d_active = dalloc<int>(16 * (size_t)H.nseg, "alloc refinement flags");
      H.d_segrow = dalloc<int>(segrow32.size(), "alloc segments");
      H.d_chunkrow = dalloc<int>(chunkrow.size(), "alloc dot chunks");
      H.d_segchunk = dalloc<int>(segchunk.size(), "alloc dot chunks");
      ck(cudaMemcpy(H.d_segrow, segrow32.data(), segrow32.size() * sizeof(int),
                    cudaMemcpyHostToDevice), "upload segments");
      ck(cudaMemcpy(H.d_chunkrow, chunkrow.data(), chunkrow.size() * sizeof(int),
                    cudaMemcpyHostToDevice), "upload dot chunks");
      ck(cudaMemcpy(H.d_segchunk, segchunk.data(), segchunk.size() * sizeof(int),
                    cudaMemcpyHostToDevice), "upload dot chunks");
    }
    H.d_val = dalloc<double>(H.nnz, "alloc CSR values");
    H.d_rp = dalloc<int>(n + 1, "alloc CSR rows");
    H.d_ci = dalloc<int>(H.nnz, "alloc CSR cols");
    H.d_dofs = dalloc<int>(s.dofs.size(), "alloc DOF table");
    std::vector<FrontDev> fr(s.fronts.size());
    std::vector<int64_t> woff(s.fronts.size() + 1, 0);
    for (size_t i = 0; i < s.fronts.size(); i++) {
      const mfgpu::Front& f = s.fronts[i];
      fr[i] = FrontDev{f.off, f.dof_off, f.n, f.m, f.N, f.ld};
      woff[i + 1] = woff[i] + 2 * (int64_t)f.N;
    }
    H.woffTotal = woff.back();
    H.lvMaxN.assign(s.levels, 0);
    H.lvMaxn.assign(s.levels, 0);
    for (const mfgpu::Front& f : s.fronts) {
      H.lvMaxN[f.level] = std::max(H.lvMaxN[f.level], f.N);
      H.lvMaxn[f.level] = std::max(H.lvMaxn[f.level], f.n);
    }
    {
      std::vector<int64_t> doff(s.fronts.size(), -1);
      int64_t cur = 0;
      const int B = mfgpu::kDinvBlock;
      for (size_t i = 0; i < s.fronts.size(); i++)
        if (H.coopSweep(s.fronts[i].level)) {
          doff[i] = cur;
          cur += (int64_t)((s.fronts[i].n + B - 1) / B) * 2 * B * B;
        }
      H.dinvElems = cur;
      H.h_dinv_off = doff;
      H.d_Dinv = dalloc<unsigned char>(std::max<int64_t>(cur, 1) * H.esz, "alloc block inverses");
      // task lists of the cooperative sweeps, per level
      std::vector<int> tab;
      H.flow.assign(s.levels, mfgpu_handle::FlowLevel());
      for (int ell = 0; ell < s.levels; ell++) {
        if (!H.coopSweep(ell)) continue;
        std::vector<int> nn, NN, fw, bw, fo;
        for (int b = 0; b < s.lv[ell].nbox; b++) {
          nn.push_back(s.fronts[s.lv[ell].front0 + b].n);
          NN.push_back(s.fronts[s.lv[ell].front0 + b].N);
        }
        mfgpu::flow_tasks(nn, NN, fw, bw, fo);
        mfgpu_handle::FlowLevel& q = H.flow[ell];
        q.fwd = (int64_t)tab.size();
        q.nfwd = (int)fw.size() / 2;
        tab.insert(tab.end(), fw.begin(), fw.end());
        q.bwd = (int64_t)tab.size();
        q.nbwd = (int)bw.size() / 2;
        tab.insert(tab.end(), bw.begin(), bw.end());
        q.flagoff = (int64_t)tab.size();
        q.nflags = fo.back();
        tab.insert(tab.end(), fo.begin(), fo.end());
        H.maxFlags = std::max(H.maxFlags, q.nflags);
        if (tab.size() % 2) tab.push_back(0);   // keep the next level's pairs 8-byte aligned
      }
      H.d_flow = dalloc<int>(std::max<size_t>(tab.size(), 2), "alloc sweep task lists");
      if (!tab.empty())
        ck(cudaMemcpy(H.d_flow, tab.data(), tab.size() * sizeof(int), cudaMemcpyHostToDevice),
           "upload sweep task lists");
      H.d_flags = dalloc<int>(std::max(H.maxFlags, 1), "alloc sweep ready flags");
      H.d_dinv_off = dalloc<int64_t>(doff.size(), "alloc block inverse offsets");
      ck(cudaMemcpy(H.d_dinv_off, doff.data(), doff.size() * sizeof(int64_t),
                    cudaMemcpyHostToDevice), "upload block inverse offsets");
    }
    std::vector<SepDev> sp(s.seps.size());
    for (size_t i = 0; i < s.seps.size(); i++) {
      const mfgpu::Sep& e = s.seps[i];
      sp[i] = SepDev{e.dof_off, e.s, e.box[0], e.box[1], e.bdpos[0], e.bdpos[1], 0};
    }
    std::vector<int> all;
    for (size_t i = 0; i < s.fronts.size(); i++) all.push_back((int)i);
    for (size_t i = 0; i < s.seps.size(); i++) all.push_back((int)i);
    H.d_fr = dalloc<FrontDev>(fr.size(), "alloc fronts");
    H.d_sp = dalloc<SepDev>(std::max<size_t>(1, sp.size()), "alloc seps");
    H.d_woff = dalloc<int64_t>(woff.size(), "alloc woff");
    H.d_err = dalloc<DevError>(1, "alloc error word");
    ck(cudaMemset(H.d_err, 0, sizeof(DevError)), "clear error word");
    H.d_slots = dalloc<unsigned char>(mfgpu::coop_slot_elems() * H.esz, "alloc diagonal slots");
    {
      int most = 1;   // fronts of the largest level (panel launches take up to kMaxPanelFronts)
      for (int ell = 0; ell < s.levels; ell++) most = std::max(most, s.lv[ell].nbox);
      H.d_pslot = dalloc<unsigned char>(mfgpu::panel_slot_bytes(most, (int)H.esz),
                                        "alloc panel diagonal slots");
    }
    H.d_gbar = dalloc<unsigned>(1, "alloc grid barrier");
    H.d_all = dalloc<int>(all.size(), "alloc id list");
    if (H.lu) H.d_ipiv = dalloc<int>(s.dofs.size(), "alloc LU pivots");
    ck(cudaMemcpy(H.d_val, val, H.nnz * sizeof(double), cudaMemcpyHostToDevice), "upload val");
    ck(cudaMemcpy(H.d_rp, row_ptr, (n + 1) * sizeof(int), cudaMemcpyHostToDevice), "upload rows");
    ck(cudaMemcpy(H.d_ci, col_ind, H.nnz * sizeof(int), cudaMemcpyHostToDevice), "upload cols");
    ck(cudaMemcpy(H.d_dofs, s.dofs.data(), s.dofs.size() * sizeof(int), cudaMemcpyHostToDevice),
       "upload dofs");
    ck(cudaMemcpy(H.d_fr, fr.data(), fr.size() * sizeof(FrontDev), cudaMemcpyHostToDevice), "upload fronts");
    if (!sp.empty())
      ck(cudaMemcpy(H.d_sp, sp.data(), sp.size() * sizeof(SepDev), cudaMemcpyHostToDevice), "upload seps");
    ck(cudaMemcpy(H.d_woff, woff.data(), woff.size() * sizeof(int64_t), cudaMemcpyHostToDevice), "upload woff");
    ck(cudaMemcpy(H.d_all, all.data(), all.size() * sizeof(int), cudaMemcpyHostToDevice), "upload ids");
    std::vector<char> dirty(s.fronts.size(), 1);
    H.buildPlan(H.full, dirty);
    H.full.upload(H.stream);
    H.device_bytes = (int64_t)(s.front_elems + s.sep_elems) * (int64_t)H.esz + H.nnz * 8 +
                     (H.nnz + n + 1) * 4 + (int64_t)s.dofs.size() * 4;
  });
  if (st != MFGPU_OK) {
    g_create_error = h->err;
    return st;
  }
  *out = h.release();
  return MFGPU_OK;
}

}  // namespace

static int factorImpl(mfgpu_handle* h, const double* val, int64_t nnz, bool device) {
  if (!h) return MFGPU_ERR_ARG;
  if (val && nnz != h->nnz)
    return fail(h, MFGPU_ERR_ARG, "values must match the pattern given at creation");
  return guarded(h, [&]() {
    h->factored = false;
    ck(cudaEventRecord(h->ev0, h->stream), "event");
    h->factorWith(val, device, h->full, true);
    ck(cudaEventRecord(h->ev1, h->stream), "event");
    h->checkDevError();
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
    h->prof.collect();
    h->stats.seconds = ms * 1e-3;
    h->stats.flops = h->full.flops;
    h->stats.fronts = h->full.nfronts;
    h->factored = true;
  });
}

int mfgpu_factor(mfgpu_handle* h) { return factorImpl(h, nullptr, 0, false); }

int mfgpu_autotune(mfgpu_handle* h, int reps, int* choices) {
  if (!h) return MFGPU_ERR_ARG;
  if (h->view) return fail(h, MFGPU_ERR_ARG, "a serving-loop view cannot be autotuned");
  if (reps < 1 || reps > 100) return fail(h, MFGPU_ERR_ARG, "reps must be in [1, 100]");
  if (h->lu) return fail(h, MFGPU_ERR_ARG, "LU handles (separator widths 2-3) have one kernel per level");
  return guarded(h, [&]() {
    h->factored = false;
    ck(cudaEventRecord(h->ev0, h->stream), "event");
    try {   // a tuning that fails part-way leaves the size rules in force
      h->dropGraphs(true, false);   // the level kernels change
      h->fullRuns = 0;
      if (h->mixed) h->autotuneT<float>(reps, choices);
      else h->autotuneT<double>(reps, choices);
      h->checkDevError();
    } catch (...) {
      h->tuned.clear();
      throw;
    }
    h->stats = mfgpu_stats{};
    h->stats.flops = h->full.flops;
    h->stats.fronts = h->full.nfronts;
    h->factored = true;
  });
}
// Host values replace the matrix: refuse a nonsymmetric one as mfgpu_create
// does (device-resident values are not checked).
static int checkSymmetric(mfgpu_handle* h, const double* val) {
  if (h->lu) return MFGPU_OK;   // widths 2-3: nonsymmetric by nature, factored by LU
  std::string where;
  if (const char* why = asymmetry(h->n, h->h_rowptr.data(), h->h_colind.data(), val, where))
    return fail(h, MFGPU_ERR_ARG, std::string(why) + where +
                                      ": this library factors symmetric positive definite matrices");
  return MFGPU_OK;
}

int mfgpu_refactor(mfgpu_handle* h, const double* val, int64_t nnz) {
  if (!h) return MFGPU_ERR_ARG;
  if (!val) return fail(h, MFGPU_ERR_ARG, "null values");
  if (nnz != h->nnz) return fail(h, MFGPU_ERR_ARG, "values must match the pattern given at creation");
  if (int st = checkSymmetric(h, val)) return st;
  return factorImpl(h, val, nnz, false);
}
int mfgpu_refactor_device(mfgpu_handle* h, const double* d_val, int64_t nnz) {
  if (!d_val) return fail(h, MFGPU_ERR_ARG, "null values");
  return factorImpl(h, d_val, nnz, true);
}

static int updateImpl(mfgpu_handle* h, const double* val, int64_t nnz, const int* mod, int nmod,
                      bool device) {
  if (!h) return MFGPU_ERR_ARG;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "Update() before Factor()");
  if (!val || nnz != h->nnz || (nmod > 0 && !mod) || nmod < 0)
    return fail(h, MFGPU_ERR_ARG, "Update(): values must match the factored pattern");
  for (int i = 0; i < nmod; i++)
    if (mod[i] < 0 || mod[i] >= h->n) return fail(h, MFGPU_ERR_ARG, "modified DOF out of range");
  if (!device)
    if (int st = checkSymmetric(h, val)) return st;
  return guarded(h, [&]() {
    const Schedule& s = *h->S;
    std::vector<char> dirty;
    const size_t ndirty = s.dirty_fronts(mod, nmod, dirty);
    ck(cudaEventRecord(h->ev0, h->stream), "event");
    const Plan* P = &h->full;
    if (ndirty < s.fronts.size()) {
      h->buildPlan(h->upd, dirty);
      h->upd.upload(h->stream);
      P = &h->upd;
    }
    h->factored = false;
    h->factorWith(val, device, *P, P == &h->full);
    ck(cudaEventRecord(h->ev1, h->stream), "event");
    h->checkDevError();
    h->factored = true;
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
    h->prof.collect();
    h->stats.seconds = ms * 1e-3;
    h->stats.flops = P->flops;
    h->stats.fronts = P->nfronts;
  });
}

int mfgpu_update(mfgpu_handle* h, const double* val, int64_t nnz, const int* mod, int nmod) {
  return updateImpl(h, val, nnz, mod, nmod, false);
}
int mfgpu_update_device(mfgpu_handle* h, const double* d_val, int64_t nnz, const int* mod,
                        int nmod) {
  return updateImpl(h, d_val, nnz, mod, nmod, true);
}

int mfgpu_profile_enable(mfgpu_handle* h, int on) {
  if (!h) return MFGPU_ERR_ARG;
  h->prof.on = on != 0;
  return MFGPU_OK;
}
int mfgpu_profile_reset(mfgpu_handle* h) {
  if (!h) return MFGPU_ERR_ARG;
  h->prof.reset();
  return MFGPU_OK;
}
int mfgpu_profile_read(const mfgpu_handle* h, int cls, int64_t* launches, double* ms,
                       double* flops, double* bytes) {
  if (!h || cls < 0 || cls >= MFGPU_KC_COUNT) return MFGPU_ERR_ARG;
  if (launches) *launches = h->prof.launches[cls];
  if (ms) *ms = h->prof.ms[cls];
  if (flops) *flops = h->prof.flops[cls];
  if (bytes) *bytes = h->prof.bytes[cls];
  return MFGPU_OK;
}
long long mfgpu_kernel_launches(void) { return mfgpu::launches_total(); }

static int solveOrApply(mfgpu_handle* h, const double* in, double* out, int nrhs, int64_t ld,
                        bool device, bool apply) {
  if (!h) return MFGPU_ERR_ARG;
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "Solve()/Apply() before Factor()");
  if (!in || !out || nrhs < 0 || ld < h->n) return fail(h, MFGPU_ERR_ARG, "bad vector arguments");
  if (nrhs == 0) return MFGPU_OK;
  return guarded(h, [&]() {
    const int chunk = 16;
    h->stats.iterations = 0;
    h->stats.residual = 0;
    h->clearErr();
    ck(cudaEventRecord(h->ev0, h->stream), "event");
    for (int c0 = 0; c0 < nrhs; c0 += chunk) {
      const int nc = std::min(chunk, nrhs - c0);
      h->ensureWork(nc);
      double* X = h->d_X;
      for (int c = 0; c < nc; c++)
        ck(cudaMemcpyAsync(X + (int64_t)c * h->n, in + (int64_t)(c0 + c) * ld, h->n * sizeof(double),
                           device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, h->stream),
           "copy rhs in");
      if (!h->prof.verbose) h->prof.begin(apply ? MFGPU_KC_APPLY : MFGPU_KC_SOLVE, h->stream);
      if (apply) h->applyChunk(X, nc);
      else h->solveChunk(X, nc);
      if (!h->prof.verbose) h->prof.end(h->stream);
      if (h->prof.on) {
        // L11 (lower) and L21 are read once forward and once backward; the
        // right-hand sides are gathered and scattered per front.
        double fl = 0, by = 0;
        for (const mfgpu::Front& f : h->S->fronts) {
          fl += 2.0 * ((double)f.n * f.n + 2.0 * f.n * f.m) * nc;
          by += 2.0 * h->esz * ((double)f.n * (f.n + 1) / 2 + (double)f.n * f.m) +
                h->esz * 4.0 * f.N * nc;
        }
        const int kc = apply ? MFGPU_KC_APPLY : MFGPU_KC_SOLVE;
        h->prof.flops[kc] += fl;
        h->prof.bytes[kc] += by;
      }
      for (int c = 0; c < nc; c++)
        ck(cudaMemcpyAsync(out + (int64_t)(c0 + c) * ld, X + (int64_t)c * h->n, h->n * sizeof(double),
                           device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, h->stream),
           "copy result out");
      if (!device) ck(cudaStreamSynchronize(h->stream), "solve");
    }
    ck(cudaEventRecord(h->ev1, h->stream), "event");
    ck(cudaEventSynchronize(h->ev1), "solve");
    h->checkDevError();
    h->prof.collect();
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
    h->stats.seconds = ms * 1e-3;
    double fl = 0;
    for (const mfgpu::Front& f : h->S->fronts) fl += 2.0 * ((double)f.n * f.n + 2.0 * f.n * f.m);
    h->stats.flops = fl * nrhs;
  });
}

int mfgpu_solve(mfgpu_handle* h, const double* b, double* x, int nrhs, int64_t ld) {
  return solveOrApply(h, b, x, nrhs, ld, false, false);
}
int mfgpu_apply(mfgpu_handle* h, const double* x, double* b, int nrhs, int64_t ld) {
  return solveOrApply(h, x, b, nrhs, ld, false, true);
}
int mfgpu_solve_device(mfgpu_handle* h, const double* b, double* x, int nrhs, int64_t ld) {
  return solveOrApply(h, b, x, nrhs, ld, true, false);
}
int mfgpu_apply_device(mfgpu_handle* h, const double* x, double* b, int nrhs, int64_t ld) {
  return solveOrApply(h, x, b, nrhs, ld, true, true);
}

// ---- solve without any device allocation ----
//
// mfgpu_solve_device grows a workspace with cudaMalloc the first time it sees
// a problem or a larger right-hand-side count.  Callers that may not allocate
// device memory at solve time (a service that reserves all device memory when
// it starts and must stay inside that budget, or a real-time loop that cannot
// afford cudaMalloc's implicit device-wide synchronisation) use this variant:
// its workspace is a fixed array compiled into the library, 32 MiB on every
// GPU that loads the library, held until the process exits.
namespace {
constexpr size_t kNoAllocScratchDoubles = size_t(4) << 20;   // 32 MiB
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on device `dev`, which must be current.
// Host code cannot use the array's name as a device pointer, so the address is
// looked up once per device and cached.
double* noallocScratch(int dev) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (dev < 0 || dev >= kNoAllocMaxDevices)
    throw CudaError("device ordinal out of range for the no-allocation scratch", MFGPU_ERR_ARG);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    ck(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(no-allocation scratch)");
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_ptr[dev];
}
}  // namespace

int mfgpu_solve_device_noalloc(mfgpu_handle* h, const double* d_b, double* d_x, int nrhs,
                               int64_t ld) {
  if (!h) return MFGPU_ERR_ARG;
  if (h->mixed)
    return fail(h, MFGPU_ERR_ARG,
                "mfgpu_solve_device_noalloc supports FP64 handles only (mixed precision refines "
                "with allocated work vectors); use mfgpu_solve_device");
  const int64_t per_rhs = h->woffTotal;   // workspace doubles one right-hand side needs
  if (per_rhs > (int64_t)kNoAllocScratchDoubles) {
    char buf[256];
    snprintf(buf, sizeof buf,
             "problem too large for mfgpu_solve_device_noalloc: one right-hand side needs %.1f MiB "
             "of workspace, the fixed scratch holds %.1f MiB; use mfgpu_solve_device",
             per_rhs * 8.0 / 1048576.0, kNoAllocScratchDoubles * 8.0 / 1048576.0);
    return fail(h, MFGPU_ERR_ARG, buf);
  }
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "Solve() before Factor()");
  if (!d_b || !d_x || nrhs < 0 || ld < h->n) return fail(h, MFGPU_ERR_ARG, "bad vector arguments");
  if (nrhs == 0) return MFGPU_OK;
  return guarded(h, [&]() {
    double* W = noallocScratch(h->device);
    const int chunk = (int)std::min<int64_t>(16, (int64_t)kNoAllocScratchDoubles / per_rhs);
    // the error word reports a cooperative sweep's grid barrier that gave up
    h->clearErr();
    ck(cudaEventRecord(h->ev0, h->stream), "event");
    for (int c0 = 0; c0 < nrhs; c0 += chunk) {
      const int nc = std::min(chunk, nrhs - c0);
      double* X = d_x + (int64_t)c0 * ld;
      if (d_x != d_b)
        for (int c = 0; c < nc; c++)
          ck(cudaMemcpyAsync(X + (int64_t)c * ld, d_b + (int64_t)(c0 + c) * ld, h->n * sizeof(double),
                             cudaMemcpyDeviceToDevice, h->stream),
             "copy rhs");
      h->solveChunkScratch(X, ld, nc, W);
    }
    ck(cudaEventRecord(h->ev1, h->stream), "event");
    h->checkDevError();   // synchronises the stream
    float ms = 0;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
    h->stats.seconds = ms * 1e-3;
    double fl = 0;
    for (const mfgpu::Front& f : h->S->fronts) fl += 2.0 * ((double)f.n * f.n + 2.0 * f.n * f.m);
    h->stats.flops = fl * nrhs;
    h->stats.iterations = 0;
    h->stats.residual = 0;
  });
}

// ---- stencil assembly on the device ----

int mfgpu_stencil_assemble_device(mfgpu_handle* h, const double* d_coef, const double* hxyz,
                                  double* d_val) {
  if (!h) return MFGPU_ERR_ARG;
  const Schedule& s = *h->S;
  if (s.forest() || s.width != 1 || !d_coef || !d_val)
    return fail(h, MFGPU_ERR_ARG,
                "stencil assembly needs one problem of width 1 and non-null pointers");
  const double hh[3] = {hxyz ? hxyz[0] : 1.0, hxyz ? hxyz[1] : 1.0, hxyz ? hxyz[2] : 1.0};
  return guarded(h, [&]() {
    const int lo[3] = {0, 0, 0}, hi[3] = {s.N[0], s.N[1], s.dim == 3 ? s.N[2] : 1};
    ck(mfgpu::launch_stencil_rows(s.dim, s.N[0], s.N[1], s.N[2], hh, d_coef, h->d_rp, d_val, lo,
                                  hi, nullptr, h->stream),
       "launch stencil assembly (k_stencil_rows)");
    ck(cudaStreamSynchronize(h->stream), "stencil assembly");
  });
}

int mfgpu_stencil_update_device(mfgpu_handle* h, const double* d_coef, const double* hxyz,
                                const int* box_lo, const int* box_hi, double* d_val,
                                int* modified_dofs, int capacity, int* n_modified) {
  if (!h) return MFGPU_ERR_ARG;
  const Schedule& s = *h->S;
  if (s.forest() || s.width != 1 || !d_coef || !d_val || !box_lo || !box_hi || !n_modified)
    return fail(h, MFGPU_ERR_ARG,
                "stencil update needs one problem of width 1 and non-null pointers");
  const double hh[3] = {hxyz ? hxyz[0] : 1.0, hxyz ? hxyz[1] : 1.0, hxyz ? hxyz[2] : 1.0};
  // rows whose stencil reads a node of the changed cells: the box grown by one
  int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  int64_t cells = 1;
  for (int a = 0; a < s.dim; a++) {
    lo[a] = std::max(0, box_lo[a] - 1);
    hi[a] = std::min(s.N[a], box_hi[a] + 1);
    if (hi[a] <= lo[a]) {
      *n_modified = 0;
      return MFGPU_OK;
    }
    cells *= hi[a] - lo[a];
  }
  return guarded(h, [&]() {
    if (!h->d_flag) h->d_flag = dalloc<int>((size_t)h->n + 1, "alloc row flags");
    h->growBuf(h->d_modbuf, h->capMod, (size_t)cells, "alloc modified rows");
    int* d_count = h->d_flag + h->n;
    ck(cudaMemsetAsync(d_count, 0, sizeof(int), h->stream), "clear count");
    ck(mfgpu::launch_stencil_rows(s.dim, s.N[0], s.N[1], s.N[2], hh, d_coef, h->d_rp, d_val, lo,
                                  hi, h->d_flag, h->stream),
       "launch stencil update (k_stencil_rows)");
    ck(mfgpu::launch_collect_rows(s.dim, s.N[0], s.N[1], lo, hi, h->d_flag, h->d_modbuf,
                                  (int)cells, d_count, h->stream),
       "launch modified-row collection (k_collect)");
    int cnt = 0;
    ck(cudaMemcpyAsync(&cnt, d_count, sizeof(int), cudaMemcpyDeviceToHost, h->stream), "read count");
    ck(cudaStreamSynchronize(h->stream), "stencil update");
    std::vector<int> rows(cnt);
    if (cnt)
      ck(cudaMemcpy(rows.data(), h->d_modbuf, cnt * sizeof(int), cudaMemcpyDeviceToHost),
         "read modified rows");
    std::sort(rows.begin(), rows.end());
    *n_modified = cnt;
    if (modified_dofs) {
      if (cnt > capacity) throw CudaError("modified-DOF buffer too small", MFGPU_ERR_ARG);
      std::copy(rows.begin(), rows.end(), modified_dofs);
    }
  });
}

int mfgpu_set_wait_limit(mfgpu_handle* h, unsigned polls) {
  if (!h) return MFGPU_ERR_ARG;
  return guarded(h, [&]() { h->setLimit(polls); });
}

int mfgpu_graphs(const mfgpu_handle* h, int* factor_graph, int* sweep_graphs) {
  if (!h) return MFGPU_ERR_ARG;
  if (factor_graph) *factor_graph = h->fullGraph ? 1 : 0;
  if (sweep_graphs) *sweep_graphs = (int)h->sweepGraphs.size();
  return MFGPU_OK;
}

void mfgpu_inject_alloc_failure(long long after) { g_alloc_budget.store(after < 0 ? -1 : after); }

int mfgpu_set_stream(mfgpu_handle* h, void* st) {
  if (!h) return MFGPU_ERR_ARG;
  return guarded(h, [&]() {
    ck(cudaStreamSynchronize(h->stream), "sync old stream");
    h->stream = st ? static_cast<cudaStream_t>(st) : h->own;
  });
}

namespace {

// Factor file: FacHeader, the payload blocks of facBlocks in order, then a
// 64-bit FNV-1a checksum of the payload (taken 8 bytes at a time).
struct FacHeader {
  char magic[8];
  uint32_t version, esz, mixed, pad;
  int64_t n, nnz, front_elems, sep_elems, dinv_elems, nfronts, nseps;
  uint64_t pattern;   // checksum of row_ptr and col_ind
};
constexpr char kFacMagic[8] = {'M', 'F', 'G', 'P', 'U', 'F', 'A', 'C'};
constexpr uint32_t kFacVersion = 1;
constexpr uint64_t kFnvBasis = 1469598103934665603ull, kFnvPrime = 1099511628211ull;

uint64_t fnv64(uint64_t h, const unsigned char* p, size_t bytes) {
  size_t i = 0;
  for (; i + 8 <= bytes; i += 8) {
    uint64_t w;
    std::memcpy(&w, p + i, 8);
    h = (h ^ w) * kFnvPrime;
  }
  for (; i < bytes; i++) h = (h ^ p[i]) * kFnvPrime;
  return h;
}

FacHeader facHeader(const mfgpu_handle* h) {
  FacHeader f;
  std::memset(&f, 0, sizeof f);
  std::memcpy(f.magic, kFacMagic, 8);
  f.version = kFacVersion;
  f.esz = (uint32_t)h->esz;
  f.mixed = h->mixed ? 1 : 0;
  f.n = h->n;
  f.nnz = h->nnz;
  f.front_elems = h->S->front_elems;
  f.sep_elems = h->S->sep_elems;
  f.dinv_elems = h->dinvElems;
  f.nfronts = (int64_t)h->S->fronts.size();
  f.nseps = (int64_t)h->S->seps.size();
  uint64_t c = fnv64(kFnvBasis, (const unsigned char*)h->h_rowptr.data(), h->h_rowptr.size() * 4);
  f.pattern = fnv64(c, (const unsigned char*)h->h_colind.data(), h->h_colind.size() * 4);
  return f;
}

// The device arrays that make up a factored handle, in file order.
std::vector<std::pair<void*, size_t>> facBlocks(const mfgpu_handle* h) {
  std::vector<std::pair<void*, size_t>> b = {{h->d_F, (size_t)h->S->front_elems * h->esz},
                                             {h->d_Sep, (size_t)h->S->sep_elems * h->esz},
                                             {h->d_val, (size_t)h->nnz * sizeof(double)}};
  if (h->mixed) {
    b.push_back({h->d_scale, (size_t)h->n * sizeof(double)});
    b.push_back({h->d_iscale, (size_t)h->n * sizeof(double)});
  }
  if (h->dinvElems > 0) b.push_back({h->d_Dinv, (size_t)h->dinvElems * h->esz});
  if (h->lu) b.push_back({h->d_ipiv, h->S->dofs.size() * sizeof(int)});
  return b;
}

struct FileCloser {
  void operator()(FILE* f) const {
    if (f) fclose(f);
  }
};

constexpr size_t kFacChunk = (size_t)64 << 20;   // host bounce buffer

}  // namespace

int mfgpu_save(mfgpu_handle* h, const char* path) {
  if (!h) return MFGPU_ERR_ARG;
  if (!path) return fail(h, MFGPU_ERR_ARG, "null path");
  if (h->view) return fail(h, MFGPU_ERR_ARG, "a serving-loop view cannot be saved");
  if (!h->factored) return fail(h, MFGPU_ERR_STATE, "save before a successful Factor()");
  return guarded(h, [&]() {
    ck(cudaStreamSynchronize(h->stream), "sync before save");
    std::unique_ptr<FILE, FileCloser> f(fopen(path, "wb"));
    if (!f) throw CudaError(std::string("cannot open ") + path + " for writing", MFGPU_ERR_ARG);
    const FacHeader hd = facHeader(h);
    if (fwrite(&hd, sizeof hd, 1, f.get()) != 1)
      throw CudaError(std::string("write failed: ") + path, MFGPU_ERR_ARG);
    std::vector<unsigned char> buf;
    uint64_t sum = kFnvBasis;
    for (const auto& blk : facBlocks(h)) {
      for (size_t o = 0; o < blk.second; o += kFacChunk) {
        const size_t len = std::min(kFacChunk, blk.second - o);
        buf.resize(len);
        ck(cudaMemcpy(buf.data(), (const unsigned char*)blk.first + o, len, cudaMemcpyDeviceToHost),
           "copy factor to host");
        sum = fnv64(sum, buf.data(), len);
        if (fwrite(buf.data(), 1, len, f.get()) != len)
          throw CudaError(std::string("write failed: ") + path, MFGPU_ERR_ARG);
      }
    }
    if (fwrite(&sum, sizeof sum, 1, f.get()) != 1 || fflush(f.get()) != 0)
      throw CudaError(std::string("write failed: ") + path, MFGPU_ERR_ARG);
  });
}

int mfgpu_load(mfgpu_handle* h, const char* path) {
  if (!h) return MFGPU_ERR_ARG;
  if (!path) return fail(h, MFGPU_ERR_ARG, "null path");
  if (h->view) return fail(h, MFGPU_ERR_ARG, "a serving-loop view cannot be loaded into");
  return guarded(h, [&]() {
    std::unique_ptr<FILE, FileCloser> f(fopen(path, "rb"));
    if (!f) throw CudaError(std::string("cannot open ") + path, MFGPU_ERR_ARG);
    FacHeader hd;
    if (fread(&hd, sizeof hd, 1, f.get()) != 1 || std::memcmp(hd.magic, kFacMagic, 8) != 0 ||
        hd.version != kFacVersion)
      throw CudaError(std::string(path) + " is not a factor file of this library version",
                      MFGPU_ERR_ARG);
    const FacHeader me = facHeader(h);
    const char* what = hd.esz != me.esz || hd.mixed != me.mixed ? "precision"
                       : hd.n != me.n || hd.nnz != me.nnz || hd.pattern != me.pattern
                           ? "matrix size or sparsity pattern"
                       : hd.front_elems != me.front_elems || hd.sep_elems != me.sep_elems ||
                               hd.dinv_elems != me.dinv_elems || hd.nfronts != me.nfronts ||
                               hd.nseps != me.nseps
                           ? "elimination-tree schedule"
                           : nullptr;
    if (what)
      throw CudaError(std::string("factor file ") + path + " does not match this handle (" + what + ")",
                      MFGPU_ERR_ARG);
    ck(cudaStreamSynchronize(h->stream), "sync before load");
    h->factored = false;
    std::vector<unsigned char> buf;
    uint64_t sum = kFnvBasis;
    for (const auto& blk : facBlocks(h)) {
      for (size_t o = 0; o < blk.second; o += kFacChunk) {
        const size_t len = std::min(kFacChunk, blk.second - o);
        buf.resize(len);
        if (fread(buf.data(), 1, len, f.get()) != len)
          throw CudaError(std::string("factor file ") + path + " is truncated", MFGPU_ERR_ARG);
        sum = fnv64(sum, buf.data(), len);
        ck(cudaMemcpy((unsigned char*)blk.first + o, buf.data(), len, cudaMemcpyHostToDevice),
           "copy factor to device");
      }
    }
    uint64_t want = 0;
    if (fread(&want, sizeof want, 1, f.get()) != 1 || want != sum)
      throw CudaError(std::string("factor file ") + path + " fails its checksum", MFGPU_ERR_ARG);
    h->stats = mfgpu_stats{};
    h->factored = true;
  });
}

int mfgpu_get_info(const mfgpu_handle* h, mfgpu_info* info) {
  if (!h || !info) return MFGPU_ERR_ARG;
  const Schedule& s = *h->S;
  std::memset(info, 0, sizeof(*info));
  info->dim = s.dim;
  info->levels = s.levels;
  info->n_fronts = (int)s.fronts.size();
  info->n_seps = (int)s.seps.size();
  info->ndof = s.ndof;
  info->nnz = h->nnz;
  for (int a = 0; a < 3; a++) info->leaf_box[a] = s.bw[a];
  for (const mfgpu::Front& f : s.fronts) info->max_front = std::max(info->max_front, f.N);
  info->factor_flops = s.total_flops();
  info->front_bytes = s.front_elems * (int64_t)h->esz;
  info->sep_bytes = s.sep_elems * (int64_t)h->esz;
  info->device_bytes = h->device_bytes;
  return MFGPU_OK;
}

int mfgpu_last_stats(const mfgpu_handle* h, mfgpu_stats* st) {
  if (!h || !st) return MFGPU_ERR_ARG;
  *st = h->stats;
  return MFGPU_OK;
}

const char* mfgpu_last_error(const mfgpu_handle* h) {
  if (!h) return g_create_error.c_str();
  return h->err.c_str();
}

void mfgpu_destroy(mfgpu_handle* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  delete h;
}

// ---- host-only symbolic access ----
struct mfgpu_symbolic {
  std::unique_ptr<Schedule> S;
};

static int symbolicCreate(int dim, int nx, int ny, int nz, int width, int max_side, bool full,
                          mfgpu_symbolic** out) {
  if (!out) return MFGPU_ERR_ARG;
  *out = nullptr;
  g_sym_error.clear();
  try {
    std::unique_ptr<mfgpu_symbolic> s(new mfgpu_symbolic());
    s->S.reset(new Schedule(dim, nx, ny, nz, width, max_side, full));
    *out = s.release();
    return MFGPU_OK;
  } catch (const std::invalid_argument& e) {
    g_sym_error = e.what();
    return MFGPU_ERR_ARG;
  } catch (const std::runtime_error& e) {
    g_sym_error = e.what();
    return std::string(e.what()).find("recursion depth") != std::string::npos ? MFGPU_ERR_DEPTH
                                                                                : MFGPU_ERR_LEAF;
  } catch (const std::bad_alloc&) {
    return MFGPU_ERR_OOM;
  }
}

int mfgpu_symbolic_create(int dim, int nx, int ny, int nz, int width, int max_side,
                          mfgpu_symbolic** out) {
  return symbolicCreate(dim, nx, ny, nz, width, max_side, false, out);
}

int mfgpu_symbolic_create_full(int dim, int nx, int ny, int nz, int width, int max_side,
                               mfgpu_symbolic** out) {
  return symbolicCreate(dim, nx, ny, nz, width, max_side, true, out);
}

int mfgpu_symbolic_batch_create(int count, const int* dim, const int* nx, const int* ny,
                                const int* nz, const int* width, const int* max_side,
                                mfgpu_symbolic** out) {
  if (!out || count <= 0 || !dim || !nx || !ny || !nz || !width || !max_side) return MFGPU_ERR_ARG;
  *out = nullptr;
  g_sym_error.clear();
  try {
    std::vector<Schedule> parts;
    parts.reserve(count);
    for (int p = 0; p < count; p++)
      parts.emplace_back(dim[p], nx[p], ny[p], nz[p], width[p], max_side[p]);
    std::unique_ptr<mfgpu_symbolic> s(new mfgpu_symbolic());
    s->S.reset(new Schedule(std::move(parts)));
    *out = s.release();
    return MFGPU_OK;
  } catch (const std::invalid_argument& e) {
    g_sym_error = e.what();
    return MFGPU_ERR_ARG;
  } catch (const std::runtime_error& e) {
    g_sym_error = e.what();
    return std::string(e.what()).find("recursion depth") != std::string::npos ? MFGPU_ERR_DEPTH
                                                                                : MFGPU_ERR_LEAF;
  } catch (const std::bad_alloc&) {
    return MFGPU_ERR_OOM;
  }
}

void mfgpu_symbolic_destroy(mfgpu_symbolic* s) { delete s; }
const char* mfgpu_symbolic_error(void) { return g_sym_error.c_str(); }

int mfgpu_symbolic_sizes(const mfgpu_symbolic* s, int* levels, int* nf, int* ns, int64_t* ndof) {
  if (!s) return MFGPU_ERR_ARG;
  if (levels) *levels = s->S->levels;
  if (nf) *nf = (int)s->S->fronts.size();
  if (ns) *ns = (int)s->S->seps.size();
  if (ndof) *ndof = s->S->ndof;
  return MFGPU_OK;
}

int mfgpu_symbolic_front(const mfgpu_symbolic* s, int f, int* level, int* box, int* n, int* m,
                         const int** dofs) {
  if (!s || f < 0 || f >= (int)s->S->fronts.size()) return MFGPU_ERR_ARG;
  const mfgpu::Front& F = s->S->fronts[f];
  if (level) *level = F.level;
  if (box) *box = F.box;
  if (n) *n = F.n;
  if (m) *m = F.m;
  if (dofs) *dofs = s->S->dofs.data() + F.dof_off;
  return MFGPU_OK;
}

int mfgpu_symbolic_sep(const mfgpu_symbolic* s, int k, int* level, int* idx, int* size,
                       const int** dofs, int boxes[2], int rows[2]) {
  if (!s || k < 0 || k >= (int)s->S->seps.size()) return MFGPU_ERR_ARG;
  const mfgpu::Sep& e = s->S->seps[k];
  if (level) *level = e.level;
  if (idx) *idx = e.idx;
  if (size) *size = e.s;
  if (dofs) *dofs = s->S->dofs.data() + e.dof_off;
  if (boxes) {
    boxes[0] = e.box[0];
    boxes[1] = e.box[1];
  }
  if (rows) {
    rows[0] = e.bdpos[0];
    rows[1] = e.bdpos[1];
  }
  return MFGPU_OK;
}

int64_t mfgpu_symbolic_tasks(const mfgpu_symbolic* s, int which, const void** tasks) {
  if (!s) return -1;
  const std::vector<Task>* v = which == 0 ? &s->S->front_tasks
                               : which == 1 ? &s->S->sep_tasks
                                            : &s->S->sep_add_tasks;
  if (tasks) *tasks = v->data();
  return (int64_t)v->size();
}

int64_t mfgpu_symbolic_dirty(const mfgpu_symbolic* s, const int* mod, int nmod,
                             unsigned char* dirty, double* flops) {
  if (!s || nmod < 0 || (nmod > 0 && !mod)) return -1;
  for (int i = 0; i < nmod; i++)
    if (mod[i] < 0 || mod[i] >= s->S->ndof) return -1;
  std::vector<char> d;
  size_t nd = s->S->dirty_fronts(mod, nmod, d);
  double fl = 0;
  for (size_t f = 0; f < d.size(); f++) {
    if (dirty) dirty[f] = (unsigned char)d[f];
    if (d[f]) fl += s->S->front_flops(s->S->fronts[f]);
  }
  if (flops) *flops = fl;
  return (int64_t)nd;
}

int mfgpu_symbolic_layout(const mfgpu_symbolic* s, int front_or_sep, int id, int64_t* off, int* ld) {
  if (!s) return MFGPU_ERR_ARG;
  if (front_or_sep == 0) {
    if (id < 0 || id >= (int)s->S->fronts.size()) return MFGPU_ERR_ARG;
    if (off) *off = s->S->fronts[id].off;
    if (ld) *ld = s->S->fronts[id].ld;
  } else {
    if (id < 0 || id >= (int)s->S->seps.size()) return MFGPU_ERR_ARG;
    if (off) *off = s->S->seps[id].off;
    if (ld) *ld = s->S->seps[id].ld;
  }
  return MFGPU_OK;
}

}  // extern "C"

// ===========================================================================
// Update-serving loop.
//
// A base factorization stays resident.  Each request changes the coefficients
// of one box of cells by a factor and brings right-hand sides; its answer is
// x = A_r^{-1} b with A_r the base matrix under that change alone, so requests
// are independent and their results do not depend on what else is in flight.
// A request refactors only the root paths of the leaves its box touches
// (src/DE/mf2d.cpp:150-181) into private copies of those fronts and
// separators, carved out of a device pool; every other front is read from the
// base factorization.  One worker thread per slot owns a view of the base
// handle (its own stream, front table, matrix values and workspaces), so
// admitted requests run concurrently on the device.  A request is admitted when
// a slot is free and the pool holds its footprint (the bytes of its private
// fronts and separators); requests wait in arrival order otherwise.
// ===========================================================================
namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  int64_t id = 0;
  int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  double factor = 1.0;
  std::vector<double> b;     // n x nrhs, column-major
  int nrhs = 0;
  double* x = nullptr;       // caller's output, n x nrhs, leading dimension ldx
  int64_t ldx = 0;
  Clock::time_point t_submit, t_start, t_done;
  int status = MFGPU_OK;
  std::string error;
  mfgpu_stats stats{};
  int64_t footprint = 0;     // pool elements
  int nfronts = 0;
  int batch = 1;             // requests served together with it (itself included)
  bool done = false;
};


inline int64_t round32(int64_t v) { return (v + 31) / 32 * 32; }

}  // namespace

// The serving loop.  One dispatcher thread takes the queued requests in
// arrival order into a batch, as many as the batch capacity and the private
// pool allow, and serves the batch with one factorization plan: every
// request's dirty root path gets private copies of its fronts and separators
// in the pool, and each tree level's assembly, partial factorization and
// separator accumulation run as the same launches for all requests of the
// batch (front copy f of batch member r is front (r + 1) * nF + f of a front
// table of (capacity + 1) * nF entries).  A level's fronts are grouped by the
// kernel each request would get alone, and no kernel's arithmetic for a front
// depends on the other fronts of its launch, so an answer is bit-identical
// alone or in any batch.  Then each request is solved with its own front
// table, values and block inverses.  Requests arriving meanwhile queue for
// the next batch.
struct mfgpu_server {
  mfgpu_handle* base = nullptr;
  double h[3] = {1.0, 1.0, 1.0};
  double* d_coef = nullptr;            // base coefficients
  int64_t coef_elems = 0;
  unsigned char* d_pool = nullptr;     // private fronts and separators
  int64_t pool_elems = 0;
  int capacity = 1;                    // requests per batch
  std::unique_ptr<mfgpu_handle> view;  // the dispatcher's handle (a view of the base)
  // batch buffers: per member coefficients, CSR values, block inverses; the
  // batch front table and block-inverse offsets
  double* d_coefB = nullptr;
  double* d_valB = nullptr;
  unsigned char* d_DinvB = nullptr;
  FrontDev* d_frB = nullptr;
  int64_t* d_dinv_offB = nullptr;
  std::thread worker;
  std::mutex mu;
  std::condition_variable cv_queue, cv_done;
  std::deque<std::shared_ptr<Request>> queue;
  std::map<int64_t, std::shared_ptr<Request>> all;
  int64_t next_id = 1;
  bool stop = false;
  std::vector<FrontDev> base_table;
  std::string err;

  ~mfgpu_server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_queue.notify_all();
    if (worker.joinable()) worker.join();
    view.reset();
    cudaFree(d_coefB);
    cudaFree(d_valB);
    cudaFree(d_DinvB);
    cudaFree(d_frB);
    cudaFree(d_dinv_offB);
    cudaFree(d_coef);
    cudaFree(d_pool);
  }

  // Private footprint of a request: the fronts refactored and the separators
  // rebuilt for its box (the box grown by one cell: every row whose stencil
  // reads a changed node).
  void dirtyOf(const Request& r, std::vector<char>& dirty, std::vector<char>& dsep,
               int64_t& elems) {
    const Schedule& s = *base->S;
    std::vector<int> mod;
    int lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    for (int a = 0; a < s.dim; a++) {
      lo[a] = std::max(0, r.lo[a] - 1);
      hi[a] = std::min(s.N[a], r.hi[a] + 1);
    }
    for (int k = lo[2]; k < hi[2]; k++)
      for (int j = lo[1]; j < hi[1]; j++)
        for (int i = lo[0]; i < hi[0]; i++)
          mod.push_back(i + j * s.N[0] + k * s.N[0] * s.N[1]);
    s.dirty_fronts(mod.data(), (int)mod.size(), dirty);
    dsep.assign(s.seps.size(), 0);
    elems = 0;
    for (size_t f = 0; f < s.fronts.size(); f++)
      if (dirty[f]) elems += round32((int64_t)s.fronts[f].ld * s.fronts[f].N);
    for (size_t k = 0; k < s.seps.size(); k++)
      if (dirty[s.seps[k].box[0]] || dirty[s.seps[k].box[1]]) {
        dsep[k] = 1;
        elems += round32((int64_t)s.seps[k].ld * s.seps[k].s);
      }
  }

  struct Member {
    std::shared_ptr<Request> r;
    std::vector<char> dirty, dsep;
    int64_t elems = 0, region = 0;
  };

  void run() {
    cudaSetDevice(base->device);
    while (true) {
      std::vector<Member> batch;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_queue.wait(lk, [&] { return stop || !queue.empty(); });
        if (stop) return;
        // admission in arrival order: while the batch has room and the pool
        // holds every admitted request's private copies
        int64_t used = 0;
        while (!queue.empty() && (int)batch.size() < capacity) {
          Member m;
          m.r = queue.front();
          dirtyOf(*m.r, m.dirty, m.dsep, m.elems);
          if (m.elems > pool_elems) {           // can never fit: refuse it alone
            if (!batch.empty()) break;
            queue.pop_front();
            m.r->status = MFGPU_ERR_OOM;
            m.r->error = "request needs more private memory than the whole pool";
            m.r->t_start = m.r->t_done = Clock::now();
            m.r->done = true;
            cv_done.notify_all();
            continue;
          }
          if (used + m.elems > pool_elems) break;
          queue.pop_front();
          m.region = used;
          m.r->footprint = m.elems;
          used += m.elems;
          batch.push_back(std::move(m));
        }
      }
      if (batch.empty()) continue;
      const Clock::time_point t0 = Clock::now();
      for (Member& m : batch) {
        m.r->t_start = t0;
        m.r->batch = (int)batch.size();
      }
      serve(batch);
      {
        std::lock_guard<std::mutex> lk(mu);
        const Clock::time_point t1 = Clock::now();
        for (Member& m : batch) {
          if (!m.r->done) m.r->t_done = t1;
          m.r->done = true;
        }
      }
      cv_done.notify_all();
    }
  }

  void serve(std::vector<Member>& batch) {
    mfgpu_handle& V = *view;
    const Schedule& s = *V.S;
    const int nF = (int)s.fronts.size();
    const int64_t nnz = V.nnz;
    FrontDev* own_fr = V.d_fr;
    double* own_val = V.d_val;
    void* own_Dinv = V.d_Dinv;
    int64_t* own_doff = V.d_dinv_off;
    auto restore = [&]() {
      V.d_fr = own_fr;
      V.d_val = own_val;
      V.d_Dinv = own_Dinv;
      V.d_dinv_off = own_doff;
    };
    const int st = guarded(&V, [&]() {
      std::vector<FrontDev> table((size_t)(batch.size() + 1) * nF);
      std::copy(base_table.begin(), base_table.end(), table.begin());
      std::vector<int64_t> doffB((size_t)(batch.size() + 1) * nF, -1);
      std::vector<BatchM> keep;
      std::vector<mfgpu_handle::BatchMember> members;
      keep.reserve(batch.size());
      for (size_t r = 0; r < batch.size(); r++) {
        Member& m = batch[r];
        Request& q = *m.r;
        double* coef = d_coefB + (int64_t)r * coef_elems;
        double* val = d_valB + (int64_t)r * nnz;
        // the request's coefficients and matrix values
        ck(cudaMemcpyAsync(coef, d_coef, coef_elems * sizeof(double), cudaMemcpyDeviceToDevice,
                           V.stream), "copy coefficients");
        ck(mfgpu::launch_scale_box(s.dim, s.N[1], s.N[2], q.lo, q.hi, q.factor, coef, V.stream),
           "launch coefficient change (k_scale_box)");
        ck(cudaMemcpyAsync(val, base->d_val, nnz * sizeof(double), cudaMemcpyDeviceToDevice,
                           V.stream), "copy values");
        int nmod = 0;
        const int rc = mfgpu_stencil_update_device(&V, coef, h, q.lo, q.hi, val, nullptr, 0, &nmod);
        if (rc != MFGPU_OK) throw CudaError(V.err, rc);
        // block inverses: the base's (the dirty fronts' are recomputed)
        if (V.dinvElems > 0)
          ck(cudaMemcpyAsync(d_DinvB + (int64_t)r * V.dinvElems * V.esz, base->d_Dinv,
                             V.dinvElems * V.esz, cudaMemcpyDeviceToDevice, V.stream),
             "copy block inverses");
        // private layout: dirty fronts then dirty separators, from the region on
        keep.emplace_back();
        BatchM& b = keep.back();
        b.poolF = ((int64_t)(d_pool - (unsigned char*)V.d_F)) / (int64_t)V.esz + m.region;
        b.poolS = ((int64_t)(d_pool - (unsigned char*)V.d_Sep)) / (int64_t)V.esz + m.region;
        b.fnew.assign(nF, -1);
        b.snew.assign(s.seps.size(), -1);
        int64_t cur = 0;
        for (int f = 0; f < nF; f++)
          if (m.dirty[f]) {
            b.fnew[f] = cur;
            cur += round32((int64_t)s.fronts[f].ld * s.fronts[f].N);
          }
        for (size_t k = 0; k < s.seps.size(); k++)
          if (m.dsep[k]) {
            b.snew[k] = cur;
            cur += round32((int64_t)s.seps[k].ld * s.seps[k].s);
          }
        FrontDev* tb = table.data() + (size_t)(r + 1) * nF;
        std::copy(base_table.begin(), base_table.end(), tb);
        int nd = 0;
        for (int f = 0; f < nF; f++) {
          if (m.dirty[f]) {
            tb[f].off = b.poolF + b.fnew[f];
            nd++;
          }
          if (V.h_dinv_off[f] >= 0)
            doffB[(size_t)(r + 1) * nF + f] = (int64_t)r * V.dinvElems + V.h_dinv_off[f];
        }
        q.nfronts = nd;
      }
      for (size_t r = 0; r < batch.size(); r++) {
        const BatchM* b = &keep[r];
        const Member* m = &batch[r];
        members.push_back(mfgpu_handle::BatchMember{
            &m->dirty, (int)(r + 1) * nF,
            [this, b, m, &s](Task& t) {
              t.dst_off = b->move(s, m->dirty, m->dsep, t.dst_arena, t.dst_off);
              if (t.kind == mfgpu::TK_COPY || t.kind == mfgpu::TK_ADD)
                t.src_off = b->move(s, m->dirty, m->dsep, t.src_arena, t.src_off);
            },
            (int64_t)r * nnz});
      }
      ck(cudaMemcpyAsync(d_frB, table.data(), table.size() * sizeof(FrontDev),
                         cudaMemcpyHostToDevice, V.stream), "upload batch front table");
      ck(cudaMemcpyAsync(d_dinv_offB, doffB.data(), doffB.size() * sizeof(int64_t),
                         cudaMemcpyHostToDevice, V.stream), "upload batch block-inverse offsets");
      V.buildPlanBatch(V.upd, members);
      V.upd.upload(V.stream);   // synchronises: the host tables above are consumed
      // one factorization of every member's private root path
      V.d_fr = d_frB;
      V.d_val = d_valB;
      V.d_Dinv = d_DinvB;
      V.d_dinv_off = d_dinv_offB;
      V.factorWith(nullptr, true, V.upd, false);
      V.checkDevError();
      restore();
    });
    restore();
    if (st != MFGPU_OK) {
      for (Member& m : batch) {
        m.r->status = st;
        m.r->error = V.err;
      }
      return;
    }
    // each member solved with its own factorization
    V.factored = true;
    for (size_t r = 0; r < batch.size(); r++) {
      Request& q = *batch[r].r;
      V.d_fr = d_frB + (size_t)(r + 1) * nF;
      V.d_val = d_valB + (int64_t)r * nnz;
      V.d_Dinv = d_DinvB + (int64_t)r * V.dinvElems * V.esz;
      std::vector<double> xs((size_t)V.n * q.nrhs);
      const int rc = solveOrApply(&V, q.b.data(), xs.data(), q.nrhs, V.n, false, false);
      restore();
      q.status = rc;
      if (rc != MFGPU_OK) {
        q.error = V.err;
      } else {
        for (int c = 0; c < q.nrhs; c++)
          std::copy(xs.begin() + (int64_t)c * V.n, xs.begin() + (int64_t)(c + 1) * V.n,
                    q.x + (int64_t)c * q.ldx);
        q.stats = V.stats;
      }
      std::lock_guard<std::mutex> lk(mu);
      q.t_done = Clock::now();
      q.done = true;
      cv_done.notify_all();
    }
  }

  // A batch member's private layout: element offsets of its front and
  // separator copies, and the map of an arena offset into them.
  struct BatchM {
    int64_t poolF = 0, poolS = 0;
    std::vector<int64_t> fnew, snew;
    int64_t move(const Schedule& s, const std::vector<char>& dirty, const std::vector<char>& dsep,
                 int16_t arena, int64_t off) const {
      if (arena == mfgpu::AR_FRONT) {
        int lo = 0, hi = (int)s.fronts.size() - 1;   // front whose storage holds off
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s.fronts[mid].off <= off) lo = mid;
          else hi = mid - 1;
        }
        return dirty[lo] ? poolF + fnew[lo] + (off - s.fronts[lo].off) : off;
      }
      int lo = 0, hi = (int)s.seps.size() - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (s.seps[mid].off <= off) lo = mid;
        else hi = mid - 1;
      }
      return dsep[lo] ? poolS + snew[lo] + (off - s.seps[lo].off) : off;
    }
  };
};

namespace {

std::unique_ptr<mfgpu_handle> makeView(mfgpu_handle& B) {
  std::unique_ptr<mfgpu_handle> V(new mfgpu_handle());
  mfgpu_handle& H = *V;
  H.view = true;
  H.S = B.S;
  H.opt = B.opt;
  H.device = B.device;
  H.n = B.n;
  H.nnz = B.nnz;
  H.d_F = B.d_F;
  H.d_Sep = B.d_Sep;
  H.d_rp = B.d_rp;
  H.d_ci = B.d_ci;
  H.d_dofs = B.d_dofs;
  H.d_sp = B.d_sp;
  H.d_woff = B.d_woff;
  H.d_all = B.d_all;
  H.mixed = B.mixed;
  H.esz = B.esz;
  H.tcMinN = B.tcMinN;
  H.tcSplit = B.tcSplit;
  H.tcSplit3Levels = B.tcSplit3Levels;
  H.tcSplitLow = B.tcSplitLow;
  H.subpanel = B.subpanel;
  H.panelMaxN = B.panelMaxN;
  H.tcSub = B.tcSub;
  H.fusedMinFronts = B.fusedMinFronts;
  H.d_scale = B.d_scale;
  H.d_iscale = B.d_iscale;
  H.nseg = B.nseg;
  H.nchunks = B.nchunks;
  H.d_segrow = B.d_segrow;
  H.d_chunkrow = B.d_chunkrow;
  H.d_segchunk = B.d_segchunk;
  H.woffTotal = B.woffTotal;
  H.lvMaxN = B.lvMaxN;
  H.lvMaxn = B.lvMaxn;
  H.solveCoopMinN = B.solveCoopMinN;
  H.stepped = B.stepped;
  ck(cudaStreamCreateWithFlags(&H.own, cudaStreamNonBlocking), "create stream");
  H.stream = H.own;
  ck(cudaEventCreate(&H.ev0), "event");
  ck(cudaEventCreate(&H.ev1), "event");
  H.d_fr = dalloc<FrontDev>(B.S->fronts.size(), "alloc view front table");
  H.d_val = dalloc<double>(B.nnz, "alloc view values");
  H.d_err = dalloc<DevError>(1, "alloc error word");
  ck(cudaMemsetAsync(H.d_err, 0, sizeof(DevError), H.stream), "clear error word");
  H.setLimit(B.waitLimit);   // the base's poll limit
  H.d_slots = dalloc<unsigned char>(mfgpu::coop_slot_elems() * H.esz, "alloc diagonal slots");
  H.d_pslot = dalloc<unsigned char>(mfgpu::panel_slot_bytes(mfgpu::kMaxPanelFronts, (int)H.esz),
                                    "alloc panel diagonal slots");
  H.d_gbar = dalloc<unsigned>(1, "alloc grid barrier");
  H.dinvElems = B.dinvElems;
  H.d_dinv_off = B.d_dinv_off;
  H.h_dinv_off = B.h_dinv_off;
  H.flow = B.flow;
  H.d_flow = B.d_flow;
  H.maxFlags = B.maxFlags;
  H.d_flags = dalloc<int>(std::max(B.maxFlags, 1), "alloc sweep ready flags");
  H.d_Dinv = dalloc<unsigned char>(std::max<int64_t>(B.dinvElems, 1) * H.esz, "alloc block inverses");
  if (H.mixed) {
    H.d_sc = dalloc<double>(80 * (size_t)H.nseg, "alloc refinement scalars");
    H.d_active = dalloc<int>(16 * (size_t)H.nseg, "alloc refinement flags");
  }
  H.factored = true;
  return V;
}

}  // namespace

extern "C" {

int mfgpu_server_create(mfgpu_handle* base, const double* d_coef, const double* hxyz, int slots,
                        int64_t pool_bytes, mfgpu_server** out) {
  if (!out || !base || !d_coef || slots <= 0 || pool_bytes <= 0) return MFGPU_ERR_ARG;
  *out = nullptr;
  const Schedule& s = *base->S;
  if (!base->factored) return fail(base, MFGPU_ERR_STATE, "the serving loop needs a factored handle");
  if (s.forest() || s.width != 1)
    return fail(base, MFGPU_ERR_ARG, "the serving loop takes one problem of width 1");
  std::unique_ptr<mfgpu_server> S(new mfgpu_server());
  S->base = base;
  S->capacity = slots;
  if (hxyz)
    for (int a = 0; a < 3; a++) S->h[a] = hxyz[a];
  const int st = guarded(base, [&]() {
    ck(cudaStreamSynchronize(base->stream), "sync base");
    S->coef_elems = (int64_t)(s.N[0] + 2) * (s.N[1] + 2) * (s.dim == 3 ? s.N[2] + 2 : 1);
    S->d_coef = dalloc<double>(S->coef_elems, "alloc server coefficients");
    ck(cudaMemcpy(S->d_coef, d_coef, S->coef_elems * sizeof(double), cudaMemcpyDeviceToDevice),
       "copy coefficients");
    S->pool_elems = pool_bytes / (int64_t)base->esz;
    S->d_pool = dalloc<unsigned char>((size_t)S->pool_elems * base->esz, "alloc server pool");
    const size_t nF = s.fronts.size();
    S->base_table.resize(nF);
    for (size_t i = 0; i < nF; i++) {
      const mfgpu::Front& f = s.fronts[i];
      S->base_table[i] = FrontDev{f.off, f.dof_off, f.n, f.m, f.N, f.ld};
    }
    S->view = makeView(*base);
    // the view's kernels read a different front table, values and block
    // inverses for every batch member, so nothing may be replayed from a graph
    S->view->graphs = false;
    S->d_coefB = dalloc<double>((size_t)slots * S->coef_elems, "alloc batch coefficients");
    S->d_valB = dalloc<double>((size_t)slots * base->nnz, "alloc batch values");
    S->d_DinvB = dalloc<unsigned char>(
        (size_t)slots * std::max<int64_t>(base->dinvElems, 1) * base->esz, "alloc batch inverses");
    S->d_frB = dalloc<FrontDev>((size_t)(slots + 1) * nF, "alloc batch front table");
    S->d_dinv_offB = dalloc<int64_t>((size_t)(slots + 1) * nF, "alloc batch inverse offsets");
  });
  if (st != MFGPU_OK) return st;
  S->worker = std::thread([srv = S.get()]() { srv->run(); });
  *out = S.release();
  return MFGPU_OK;
}

int mfgpu_server_submit(mfgpu_server* srv, const int* box_lo, const int* box_hi, double factor,
                        const double* b, int nrhs, int64_t ld, double* x, int64_t* ticket) {
  if (!srv || !box_lo || !box_hi || !b || !x || !ticket || nrhs <= 0) return MFGPU_ERR_ARG;
  const Schedule& s = *srv->base->S;
  if (ld < s.ndof) return MFGPU_ERR_ARG;
  auto r = std::make_shared<Request>();
  for (int a = 0; a < 3; a++) {
    r->lo[a] = a < s.dim ? box_lo[a] : 0;
    r->hi[a] = a < s.dim ? box_hi[a] : 1;
    if (a < s.dim && (r->lo[a] < 0 || r->hi[a] > s.N[a] || r->lo[a] >= r->hi[a]))
      return MFGPU_ERR_ARG;
  }
  r->factor = factor;
  r->nrhs = nrhs;
  r->b.resize((size_t)s.ndof * nrhs);
  for (int c = 0; c < nrhs; c++)
    std::copy(b + (int64_t)c * ld, b + (int64_t)c * ld + s.ndof, r->b.begin() + (int64_t)c * s.ndof);
  r->x = x;
  r->ldx = ld;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    r->id = srv->next_id++;
    srv->all[r->id] = r;
    srv->queue.push_back(r);
  }
  srv->cv_queue.notify_one();
  *ticket = r->id;
  return MFGPU_OK;
}

int mfgpu_server_wait(mfgpu_server* srv, int64_t ticket, mfgpu_request_info* info) {
  if (!srv) return MFGPU_ERR_ARG;
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->all.find(ticket);
    if (it == srv->all.end()) return MFGPU_ERR_ARG;
    r = it->second;
    srv->cv_done.wait(lk, [&] { return r->done; });
    srv->all.erase(it);
  }
  if (info) {
    std::memset(info, 0, sizeof(*info));
    info->status = r->status;
    const auto us = [](Clock::duration d) {
      return std::chrono::duration<double>(d).count();
    };
    info->queued_seconds = us(r->t_start - r->t_submit);
    info->latency_seconds = us(r->t_done - r->t_submit);
    info->fronts = r->nfronts;
    info->batch = r->batch;
    info->pool_bytes = r->footprint * (int64_t)srv->base->esz;
    info->iterations = r->stats.iterations;
    info->residual = r->stats.residual;
  }
  if (r->status != MFGPU_OK) srv->err = r->error;
  return r->status;
}

const char* mfgpu_server_last_error(const mfgpu_server* srv) { return srv ? srv->err.c_str() : ""; }

void mfgpu_server_destroy(mfgpu_server* srv) { delete srv; }

}  // extern "C"
