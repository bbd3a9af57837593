// engine.cu -- device engine of libqb: packs prepared systems into one batch
// on the GPU and runs md_run's step loop (src/q6/md.f90:4003-4175) with the
// kernels of kernels.cuh.  Batch entry points of the C ABI (include/qb.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "fep.hpp"
#include "kernels.cuh"
#include "qsystem.hpp"

namespace qb {
void set_error(const std::string &m);

#define CUDA_TRY(call)                                                                     \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) ::qb::fail(QB_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

template <class T>
T *dev_upload(const std::vector<T> &h, std::vector<void *> &owned) {
  size_t n = std::max<size_t>(h.size(), 1);
  T *p = nullptr;
  CUDA_TRY(cudaMalloc(&p, n * sizeof(T)));
  owned.push_back(p);
  if (!h.empty()) CUDA_TRY(cudaMemcpy(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
  else CUDA_TRY(cudaMemset(p, 0, sizeof(T)));
  return p;
}

template <class T>
T *dev_alloc(size_t n, std::vector<void *> &owned) {
  n = std::max<size_t>(n, 1);
  T *p = nullptr;
  CUDA_TRY(cudaMalloc(&p, n * sizeof(T)));
  owned.push_back(p);
  CUDA_TRY(cudaMemset(p, 0, n * sizeof(T)));
  return p;
}

// A pair of timing events, destroyed on every exit path (a failed CUDA call
// throws out of the timed loops).
struct EventPair {
  cudaEvent_t e[2] = {nullptr, nullptr};
  EventPair() {
    for (auto &x : e) {
      cudaError_t r = cudaEventCreate(&x);
      if (r != cudaSuccess) {
        x = nullptr;
        release();
        fail(QB_ERR_CUDA, std::string("cudaEventCreate: ") + cudaGetErrorString(r));
      }
    }
  }
  ~EventPair() { release(); }
  void release() {
    for (auto &x : e)
      if (x) { cudaEventDestroy(x); x = nullptr; }
  }
  EventPair(const EventPair &) = delete;
  EventPair &operator=(const EventPair &) = delete;
};

struct KernelStat { double ms = 0; long long launches = 0; };

struct Batch {
  int nsys = 0;
  qb_options opt{};
  std::vector<const System *> systems;
  std::vector<qb_sysview> views;
  std::vector<SysDev> sysh;
  DevPtrs P{};
  std::vector<void *> owned;
  cudaStream_t stream = nullptr;
  int NB = 1;
  long long istep = 0;
  int max_natom = 0, max_lrf_blocks = 1, max_nsol = 0, max_nwat = 0, max_ncgp = 0, max_ncgp_sol = 0, max_terms = 0, max_pp = 0, max_ncgp_sol_w = 0, max_qp = 0;
  bool any_any_atom = false;   // a system with any-atom charge-group cut-offs (iuse_switch_atom 0)
  // periodic box: any system in a box, putting molecules back, at constant pressure
  bool any_box = false, any_put = false, any_npt = false;
  // per system: randm's sequence (md.f90:14408, shared with the Maxwell
  // velocities) and the volume moves tried and accepted (md.f90:15812-15816)
  struct McState { bool started = false; int irand = 0; long long tries = 0, accepted = 0; };
  std::vector<McState> mc;
  int ww_wpb = WW_WPB;          // waters per block of the water-water kernels
  int max_nshell = 0;           // polarisation shells of the batch's systems, at most
  // the water pass takes a thread per water atom when that many threads
  // still fit on the GPU at once (small batches), else one per water
  bool water_atom_threads = false;
  // every system is solute atoms then 3-atom waters, and some system has
  // waters: the water pass writes the whole gradient (no memset)
  bool water_pass_zeroes = false;
  long long ww_tiles_cap = 0;   // their tile buffer's entries (32 waters per block)
  bool any_lrf = false, any_q = false, any_shake = false, any_wpol = false, any_prestr = false, any_qq = false,
       any_qb = false, any_hlj = false;
  // run-time choices the autotuner sets (qb_tuning): LRF source tiles per
  // block, water-water staging chunk (>= ww_chunk_floor, for which ww_sp is
  // sized), side streams on or off
  int ww_chunk_floor = 32, ww_chunk_max = 32;
  bool streams_on = true;
  std::vector<int2> lrf_dims;   // per system with LRF: (charge groups, source tiles)
  size_t watpol_smem = 0;
  int q_states = 0;           // state count shared by every system with Q atoms (0: they differ)
  int max_nq = 0;
  // profiling
  bool profiling = false;
  std::vector<std::pair<std::string, std::pair<cudaEvent_t, cudaEvent_t>>> pending;
  std::vector<cudaEvent_t> event_pool;
  std::map<std::string, KernelStat> stats;
  std::vector<std::string> order;
  double workload[QB_WORKLOAD_N] = {};

  // page-locked staging of the batched host copies (qb_batch_*_all)
  void *pinned = nullptr;
  size_t pinned_bytes = 0;
  void *staging(size_t bytes) {
    if (bytes > pinned_bytes) {
      if (pinned) cudaFreeHost(pinned);
      pinned = nullptr;
      pinned_bytes = 0;
      CUDA_TRY(cudaMallocHost(&pinned, bytes));
      pinned_bytes = bytes;
    }
    return pinned;
  }

  ~Batch() {
    if (stream) cudaStreamSynchronize(stream);
    if (pinned) cudaFreeHost(pinned);
    drop_graphs();
    for (int k = 0; k < 2; k++) {
      if (side[k]) { cudaStreamSynchronize(side[k]); cudaStreamDestroy(side[k]); }
      if (ev_join[k]) cudaEventDestroy(ev_join[k]);
    }
    if (ev_fork) cudaEventDestroy(ev_fork);
    for (auto &e : event_pool) cudaEventDestroy(e);
    for (auto &pe : pending) { cudaEventDestroy(pe.second.first); cudaEventDestroy(pe.second.second); }
    for (void *p : owned) cudaFree(p);
    if (stream) cudaStreamDestroy(stream);
  }

  cudaEvent_t take_event() {
    if (!event_pool.empty()) { auto e = event_pool.back(); event_pool.pop_back(); return e; }
    cudaEvent_t e;
    CUDA_TRY(cudaEventCreate(&e));
    return e;
  }

  long long launches = 0;

  template <class F>
  void launch(const char *name, F &&f) {
    launches++;
    if (!profiling) { f(); return; }
    cudaEvent_t a = take_event(), b = take_event();
    CUDA_TRY(cudaEventRecord(a, stream));
    f();
    CUDA_TRY(cudaEventRecord(b, stream));
    pending.push_back({name, {a, b}});
    if (pending.size() > 4096) collect();
  }

  void collect() {
    CUDA_TRY(cudaStreamSynchronize(stream));
    for (auto &pe : pending) {
      float ms = 0;
      cudaEventElapsedTime(&ms, pe.second.first, pe.second.second);
      auto it = stats.find(pe.first);
      if (it == stats.end()) { order.push_back(pe.first); it = stats.emplace(pe.first, KernelStat{}).first; }
      it->second.ms += ms;
      it->second.launches++;
      event_pool.push_back(pe.second.first);
      event_pool.push_back(pe.second.second);
    }
    pending.clear();
  }

  void check_launch(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(QB_ERR_CUDA, std::string("launch of ") + what + ": " + cudaGetErrorString(e));
  }

  static int cdiv(long long a, long long b) { return (int)std::max<long long>(1, (a + b - 1) / b); }

  // Pair lists and LRF multipoles of the systems due at this step
  // (force: every system, as the post-loop rebuild).
  // put: molecules of periodic boxes go back into the box first at the list
  // steps (md_run, md.f90:4009-4013).
  void build_lists(int force, bool put = false) {
    DevPtrs &p = P;
    dim3 b256(256);
    // main: Q-atom and solute lists; side 0: group centres and LRF multipoles;
    // side 1: water-water list
    cudaStream_t s1 = forking() ? side[0] : stream, s2 = forking() ? side[1] : stream;
    if (put && any_put) launch("put_back_in_box", [&] { k_put_back_in_box<<<nsys, 256, 0, stream>>>(p); });
    launch("lists_begin", [&] { k_lists_begin<<<cdiv(nsys, 128), 128, 0, stream>>>(p, force); });
    // group centres and radii first: the LRF gather and the any-atom list
    // tests read them
    if (any_lrf || any_any_atom)
      launch("cgp_centers", [&] { k_cgp_centers<<<cdiv(p.ncgp_tot, 256), b256, 0, stream>>>(p, force); });
    fork_streams();
    if (any_lrf) {
      launch("lrf_gather", [&] {
        if (opt.precision == QB_MIXED && any_box)
          k_lrf_gather_x2<true><<<dim3(max_lrfx_blocks, nsys), LRFX_BLOCK, 0, s1>>>(p, force);
        else if (opt.precision == QB_MIXED)
          k_lrf_gather_x2<false><<<dim3(max_lrfx_blocks, nsys), LRFX_BLOCK, 0, s1>>>(p, force);
        else
          k_lrf_gather<false><<<dim3(max_lrf_blocks, nsys), LRF_BLOCK, 0, s1>>>(p, force);
      });
    }
    if (max_nwat > 0)
      launch("list_ww", [&] { k_list_ww<<<dim3(cdiv(max_nwat, WL_WPB), nsys), WL_BLOCK, 0, s2>>>(p, force); });
    if (max_ncgp_sol > 0) {
      launch("list_pp", [&] { k_list_pp<<<dim3(max_ncgp_sol, nsys), 128, 0, stream>>>(p, force); });
      if (max_nwat > 0) launch("list_pw", [&] { k_list_pw<<<dim3(cdiv(max_ncgp_sol, 4), nsys), 128, 0, stream>>>(p, force); });
    }
    // a volume move rebuilds the LRF and the solute and water lists, not the
    // Q-atom lists (md.f90:15734-15744)
    if (any_q && force != 2) {
      launch("list_qp", [&] { k_list_qp<<<nsys, 256, 0, stream>>>(p, force); });
      if (max_nwat > 0) launch("list_qw", [&] { k_list_qw<<<nsys, 256, 0, stream>>>(p, force); });
    }
    join_streams();
    launch("lists_end", [&] { k_lists_end<<<cdiv(nsys, 128), 128, 0, stream>>>(p, force); });
    check_launch("list kernels");
  }

  bool lists_due() const {
    for (auto &S : sysh)
      if (istep % S.NB == 0) return true;
    return false;
  }

  // Side streams of the force fork: after the water pass the force kernels of
  // a step (all adding with atomics) run on three streams and join before the
  // leap-frog.  Profiling keeps them on the main stream, one at a time.
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t ev_fork = nullptr, ev_join[2] = {nullptr, nullptr};

  void make_side_streams() {
    for (int k = 0; k < 2; k++) {
      CUDA_TRY(cudaStreamCreateWithFlags(&side[k], cudaStreamNonBlocking));
      CUDA_TRY(cudaEventCreateWithFlags(&ev_join[k], cudaEventDisableTiming));
    }
    CUDA_TRY(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
  }

  // Fork the side streams off the main stream / join them back (no-ops when
  // profiling or without side streams).
  bool forking() const { return !profiling && side[0] && streams_on; }

  int max_lrfx_blocks = 1;   // the packed (two targets per thread) gather's grid
  void set_lrf_tpb(int tpb) {
    P.lrf_tpb = tpb;
    max_lrf_blocks = max_lrfx_blocks = 1;
    for (const int2 &d : lrf_dims) {
      max_lrf_blocks = std::max(max_lrf_blocks, cdiv(d.x, LRF_BLOCK) * cdiv(d.y, tpb));
      max_lrfx_blocks = std::max(max_lrfx_blocks, cdiv(d.x, LRFX_TARGETS) * cdiv(d.y, tpb));
    }
  }
  void fork_streams() {
    if (!forking()) return;
    CUDA_TRY(cudaEventRecord(ev_fork, stream));
    for (int k = 0; k < 2; k++) CUDA_TRY(cudaStreamWaitEvent(side[k], ev_fork, 0));
  }
  void join_streams() {
    if (!forking()) return;
    for (int k = 0; k < 2; k++) {
      CUDA_TRY(cudaEventRecord(ev_join[k], side[k]));
      CUDA_TRY(cudaStreamWaitEvent(stream, ev_join[k], 0));
    }
  }

  // Steps whose energies are recorded (output or energy-file records of any
  // system, as k_finish decides) evaluate every term's energy.  The mixed
  // engine evaluates the water-water pairs of those steps in FP64 and, on the
  // other steps, their forces alone in packed FP32.
  bool energy_due() const {
    for (auto &S : sysh) {
      if (S.iout > 0 && istep % S.iout == 0) return true;
      if (S.iene > 0 && istep > 0 && istep % S.iene == 0) return true;
    }
    return false;
  }

  // ene = 0 only on steps that record no energies (the mixed engine's
  // water-water forces then skip their energies); the FP64 engine always
  // evaluates them.
  void pot_energy(int ene = 1) {
    DevPtrs &p = P;
    const bool mixed = opt.precision == QB_MIXED;
    const bool fast_ww = mixed && !ene;
    // the water pass stores every water gradient and zeroes the solute's
    if (!water_pass_zeroes) CUDA_TRY(cudaMemsetAsync(p.d, 0, sizeof(double4) * (size_t)p.natoms_tot, stream));
    CUDA_TRY(cudaMemsetAsync(p.E, 0, sizeof(double) * QB_NE * (size_t)nsys, stream));
    CUDA_TRY(cudaMemsetAsync(p.EQ, 0, sizeof(double) * MAXS * QB_NEQ * (size_t)nsys, stream));
    // waters first: their records, and their per-atom terms as the first
    // gradient contribution (plain stores after the zeroing)
    if (max_nwat > 0) {
      if (water_atom_threads) {
        dim3 gp(cdiv(std::max(3 * max_nwat, max_nsol), 256), nsys);
        if (fast_ww) launch("pack_waters", [&] { k_pack_water_atoms<true><<<gp, 256, 0, stream>>>(p); });
        else launch("pack_waters", [&] { k_pack_water_atoms<false><<<gp, 256, 0, stream>>>(p); });
      } else if (p.n_pk_tiles > 0) {
        const int gp = p.n_pk_tiles;
        if (fast_ww) launch("pack_waters", [&] { k_pack_waters<true><<<gp, 256, 0, stream>>>(p); });
        else launch("pack_waters", [&] { k_pack_waters<false><<<gp, 256, 0, stream>>>(p); });
      }
    }
    cudaStream_t s1 = forking() ? side[0] : stream, s2 = forking() ? side[1] : stream;
    fork_streams();
    // solute terms in one launch (nonbond_pp, nonbond_qp, bonded, nonbond_qq,
    // Q bonded, restraints)
    {
      SoluteGrid G{};
      // pair blocks per system: enough for a large solute to fill the SMs
      // when the batch is small (1184 = 8 blocks per SM over the batch)
      const int cap = std::max(8, 1184 / std::max(nsys, 1));
      G.pp = max_pp > 0 ? std::min(cdiv(max_pp, 256), cap) : 0;
      G.qp = any_q && max_qp > 0 ? std::min(cdiv(max_qp, 256), cap) : 0;
      G.bonded = max_terms > 0 ? cdiv(max_terms, 256) : 0;
      G.qq = any_qq ? 1 : 0;
      G.qb = any_qb ? 1 : 0;
      G.pre = any_prestr ? 1 : 0;
      const int nb = G.pp + G.qp + G.bonded + G.qq + G.qb + G.pre;
      if (nb > 0)
        launch("solute_terms", [&] {
          dim3 g(nb, nsys);
          switch (q_states) {
            case 1: k_solute_terms<1><<<g, 256, 0, s1>>>(p, G); break;
            case 2: k_solute_terms<2><<<g, 256, 0, s1>>>(p, G); break;
            case 3: k_solute_terms<3><<<g, 256, 0, s1>>>(p, G); break;
            case 4: k_solute_terms<4><<<g, 256, 0, s1>>>(p, G); break;
            default: k_solute_terms<0><<<g, 256, 0, s1>>>(p, G);
          }
        });
    }
    if (p.n_pw_groups > 0)
      launch("nb_pw", [&] {
        const dim3 g(p.n_pw_groups, cdiv(p.pwg_cap, PW_BLOCK));
        if (fast_ww) k_nb_pw<true><<<g, PW_BLOCK, 0, s1>>>(p);
        else k_nb_pw<false><<<g, PW_BLOCK, 0, s1>>>(p);
      });
    if (max_nwat > 0) {
      dim3 gw(p.n_ww_tiles, 1);
      const int wpb = ww_wpb;
      size_t smem = (size_t)p.ww_chunk * (fast_ww ? WatRec<true>::words : WatRec<false>::words) * sizeof(float4);
      // hydrogen LJ: the whole batch takes the variant (exact zeros for systems without)
      if (fast_ww && any_hlj) {
        launch("nb_ww", [&] { k_nb_ww<true, true><<<gw, WW_BLOCK, smem, stream>>>(p, wpb); });
      } else if (fast_ww) {
        launch("nb_ww_x2", [&] {
          if (any_box) k_nb_ww_x2<true><<<gw, WWX_BLOCK, smem, stream>>>(p, wpb);
          else k_nb_ww_x2<false><<<gw, WWX_BLOCK, smem, stream>>>(p, wpb);
        });
      } else if (any_hlj) {
        launch("nb_ww", [&] { k_nb_ww<false, true><<<gw, WW_BLOCK, smem, stream>>>(p, wpb); });
      } else if (mixed) {
        // a recording step of the mixed engine: the packed kernel's forces,
        // the energies in FP64 over each pair once
        const size_t smem32 = (size_t)p.ww_chunk * WatRec<true>::words * sizeof(float4);
        launch("nb_ww_x2", [&] {
          if (any_box) k_nb_ww_x2<true><<<gw, WWX_BLOCK, smem32, stream>>>(p, wpb);
          else k_nb_ww_x2<false><<<gw, WWX_BLOCK, smem32, stream>>>(p, wpb);
        });
        launch("nb_ww", [&] { k_nb_ww<false, false, true><<<gw, WW_BLOCK, smem, stream>>>(p, wpb); });
      } else {
        launch("nb_ww", [&] { k_nb_ww<false, false><<<gw, WW_BLOCK, smem, stream>>>(p, wpb); });
      }
      if (any_q && p.n_qw_tiles > 0) launch("nb_qw", [&] {
        const int g = p.n_qw_tiles;
        if (any_hlj) {   // hydrogen LJ: the generic state count only
          if (max_nq > NQ_SHARED) k_nb_qw<0, false, true><<<g, 128, 0, s2>>>(p);
          else k_nb_qw<0, true, true><<<g, 128, 0, s2>>>(p);
          return;
        }
        if (max_nq > NQ_SHARED) { k_nb_qw<0, false, false><<<g, 128, 0, s2>>>(p); return; }
        // the mixed engine's non-recording steps: forces alone in FP32
        if (fast_ww) {
          switch (q_states) {
            case 1: k_nb_qw<1, true, false, true><<<g, 128, 0, s2>>>(p); break;
            case 2: k_nb_qw<2, true, false, true><<<g, 128, 0, s2>>>(p); break;
            default: k_nb_qw<0, true, false, true><<<g, 128, 0, s2>>>(p);
          }
          return;
        }
        switch (q_states) {
          case 1: k_nb_qw<1, true, false><<<g, 128, 0, s2>>>(p); break;
          case 2: k_nb_qw<2, true, false><<<g, 128, 0, s2>>>(p); break;
          case 3: k_nb_qw<3, true, false><<<g, 128, 0, s2>>>(p); break;
          case 4: k_nb_qw<4, true, false><<<g, 128, 0, s2>>>(p); break;
          default: k_nb_qw<0, true, false><<<g, 128, 0, s2>>>(p);
        }
      });
    }
    if (max_nsol > 0)
      launch("atom_terms", [&] { k_atom_terms<<<dim3(cdiv(max_nsol, 128), nsys), 128, 0, s1>>>(p); });
    if (any_wpol) {
      launch("watpol_rank", [&] { k_watpol_rank<<<dim3(std::max(max_nshell, 1), nsys), WPOL_BLOCK, watpol_smem, s2>>>(p); });
      if (p.n_wp_tiles > 0)
        launch("watpol", [&] { k_watpol_force<<<p.n_wp_tiles, WPOL_BLOCK, 0, s2>>>(p); });
    }
    join_streams();
    check_launch("force kernels");
  }

  // CUDA graphs of one step, with and without the list rebuild; kernel
  // arguments are captured by value, so any change of P drops them.
  // CUDA graphs of one step: [list rebuild][energies recorded]
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  long long graph_launches[2][2] = {{0, 0}, {0, 0}};
  bool use_graphs = true;
  // the last step of a run evaluates energies, so that the energies a caller
  // reads after it are complete
  bool force_energy = false;

  void drop_graphs() {
    for (auto &row : graph)
      for (auto &g : row)
        if (g) { cudaGraphExecDestroy(g); g = nullptr; }
    for (auto &c : cycle_graphs) cudaGraphExecDestroy(c.second.first);
    cycle_graphs.clear();
  }

  // Graphs of a whole list cycle: NB steps from a rebuild step, captured
  // once per pattern of energy-recording steps (bit k + 1: step k records;
  // bit 0: the run ends with the cycle) and
  // replayed as one launch.  Used when every system shares one non-bond
  // interval of at most 62 steps and no volume moves interrupt the cycle.
  std::map<unsigned long long, std::pair<cudaGraphExec_t, long long>> cycle_graphs;
  bool cycle_ok() const {
    if (!use_graphs || profiling || any_npt || NB > 62 || NB < 2) return false;
    for (auto &S : sysh)
      if (S.NB != NB) return false;
    return true;
  }

  // nsteps >= NB steps from a rebuild step as one cycle graph; `last`: the
  // cycle's last step is the run's last (it evaluates energies)
  void cycle(bool last) {
    unsigned long long key = last ? 1ull : 0ull;
    const long long i0 = istep;
    for (int k = 0; k < NB; k++) {
      istep = i0 + k;
      const int ene = (opt.precision != QB_MIXED || energy_due() || (last && k == NB - 1)) ? 1 : 0;
      if (ene) key |= 2ull << k;
    }
    istep = i0;
    auto it = cycle_graphs.find(key);
    if (it == cycle_graphs.end()) {
      cudaGraph_t g = nullptr;
      long long l0 = launches;
      CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      try {
        for (int k = 0; k < NB; k++) {
          istep = i0 + k;
          const int ene = (key >> (k + 1)) & 1ull;
          step_kernels(k == 0 ? 1 : 0, ene);
        }
      } catch (...) {
        istep = i0;
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      istep = i0;
      CUDA_TRY(cudaStreamEndCapture(stream, &g));
      cudaGraphExec_t ge = nullptr;
      cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) fail(QB_ERR_CUDA, std::string("graph instantiation: ") + cudaGetErrorString(e));
      it = cycle_graphs.emplace(key, std::make_pair(ge, launches - l0)).first;
      launches = l0;
    }
    CUDA_TRY(cudaGraphLaunch(it->second.first, stream));
    launches += it->second.second;
    istep = i0 + NB;
  }

  bool lists_stale = false;

  void step() {
    int due = lists_due() ? 1 : 0;
    if (lists_stale) {
      build_lists(1, true);
      lists_stale = false;
      due = 0;
    }
    const int ene = (opt.precision != QB_MIXED || force_energy || energy_due()) ? 1 : 0;
    if (!use_graphs || profiling) { step_kernels(due, ene); istep++; return; }
    cudaGraphExec_t &ge = graph[due][ene];
    if (!ge) {
      cudaGraph_t g = nullptr;
      long long l0 = launches;
      CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      try {
        step_kernels(due, ene);
      } catch (...) {
        cudaStreamEndCapture(stream, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      CUDA_TRY(cudaStreamEndCapture(stream, &g));
      cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) { ge = nullptr; fail(QB_ERR_CUDA, std::string("graph instantiation: ") + cudaGetErrorString(e)); }
      graph_launches[due][ene] = launches - l0;
      launches = l0;
    }
    CUDA_TRY(cudaGraphLaunch(ge, stream));
    launches += graph_launches[due][ene];
    istep++;
  }

  // nsteps steps, the last of them with energies
  void steps(int nsteps) {
    const bool cyc = cycle_ok();
    for (int k = 0; k < nsteps;) {
      // whole list cycles as one graph launch each, single steps elsewhere
      if (cyc && !lists_stale && istep % NB == 0 && nsteps - k >= NB) {
        cycle(k + NB == nsteps);
        k += NB;
        continue;
      }
      force_energy = k == nsteps - 1;
      step();
      if (any_npt) mc_volume(istep - 1);
      k++;
    }
    force_energy = false;
  }

  // randm (md.f90:14408-14442): the system's one sequence, seeded by the
  // first call's argument
  static double randm(McState &m, int seed) {
    const int M = 100000000, M1 = 10000, MULT = 31415821;
    if (!m.started) { m.started = true; m.irand = std::abs(seed) % M; }
    const int ih = m.irand / M1, il = m.irand % M1;
    int r = ((ih * (MULT % M1) + il * (MULT / M1)) % M1) * M1 + il * (MULT % M1);
    r = (r + 1) % M;
    m.irand = r;
    float v = (float)(r / 10) * 10.0f / (float)M;
    if (v <= 0.0f || v > 1.0f) v = 0.0f;
    return (double)v;
  }

  // new_potential's total (md.f90:15968-15971): the bonded terms of the
  // step's energies `old` with the nonbonded, restraint and LRF terms of `e`
  static double new_potential(const double *old, const double *e) {
    return old[QB_E_P_BOND] + old[QB_E_W_BOND] + old[QB_E_P_ANGLE] + old[QB_E_W_ANGLE] + old[QB_E_P_TORSION] +
           old[QB_E_P_IMPROPER] + e[QB_E_PP_EL] + e[QB_E_PP_VDW] + e[QB_E_PW_EL] + e[QB_E_PW_VDW] + e[QB_E_WW_EL] +
           e[QB_E_WW_VDW] + old[QB_E_Q_BOND] + old[QB_E_Q_ANGLE] + old[QB_E_Q_TORSION] + old[QB_E_Q_IMPROPER] +
           e[QB_E_QX_EL] + e[QB_E_QX_VDW] + e[QB_E_RST_PROTEIN] + e[QB_E_LRF];
  }

  // Energies of the current coordinates as new_potential takes them: the full
  // evaluation (the lists as they stand), summed; E and EQ copied out.
  void evaluate_into(std::vector<double> &E, std::vector<double> &EQ) {
    pot_energy(1);
    k_finish<<<nsys, 32, 0, stream>>>(P, 2);
    check_launch("energy sums");
    E.resize((size_t)nsys * QB_NE);
    EQ.resize((size_t)nsys * MAXS * QB_NEQ);
    CUDA_TRY(cudaMemcpyAsync(E.data(), P.E, sizeof(double) * E.size(), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaMemcpyAsync(EQ.data(), P.EQ, sizeof(double) * EQ.size(), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
  }

  // MC_volume (md.f90:15615-15840) after step `done` for every system at
  // constant pressure whose volume_change interval divides it: the energy of
  // the current coordinates, a random volume change, every molecule's centre
  // of mass scaled with the box, the LRF and the solute and water lists
  // rebuilt (with LRF), the energy again, and Metropolis acceptance of
  // dW = dE + p dV - N kT ln(V'/V); a rejected move restores coordinates, box
  // and LRF.  The energies that step records (output, energy file) become
  // the accepted configuration's, as the reference writes E and EQ after the
  // move.  Runs on the host between graph launches, with the device
  // evaluations batched over all systems.
  void mc_volume(long long done) {
    std::vector<int> M;
    for (int s = 0; s < nsys; s++) {
      const qb_sysview &V = views[s];
      if (V.use_pbc && V.constant_pressure && V.ivolume_cycle > 0 && done > 0 && done % V.ivolume_cycle == 0)
        M.push_back(s);
    }
    if (M.empty()) return;
    if (mc.size() != (size_t)nsys) mc.resize(nsys);
    std::vector<SysState> st(nsys);
    CUDA_TRY(cudaMemcpyAsync(st.data(), P.st, sizeof(SysState) * nsys, cudaMemcpyDeviceToHost, stream));
    // the step's energies: bonded terms of the totals, and what every other
    // system keeps
    std::vector<double> E0((size_t)nsys * QB_NE), EQ0((size_t)nsys * MAXS * QB_NEQ);
    CUDA_TRY(cudaMemcpyAsync(E0.data(), P.E, sizeof(double) * E0.size(), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaMemcpyAsync(EQ0.data(), P.EQ, sizeof(double) * EQ0.size(), cudaMemcpyDeviceToHost, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));
    std::vector<int> live;
    for (int s : M)
      if (st[s].status == 0) live.push_back(s);
    if (live.empty()) return;
    // first new_potential: the coordinates after the step
    std::vector<double> E1, EQ1, E2, EQ2;
    evaluate_into(E1, EQ1);
    // backups of the moving systems: coordinates and LRF records
    const size_t ax = (size_t)P.natoms_tot, lx = (size_t)P.ncgp_tot * LRF_STRIDE;
    if (!mc_x) {
      mc_x = dev_alloc<double4>(ax, owned);
      mc_lrf = dev_alloc<double>(std::max<size_t>(lx, 1), owned);
    }
    std::vector<double> dV(nsys, 0.0), oldV(nsys, 0.0);
    for (int s : live) {
      const SysDev &S = sysh[s];
      const qb_sysview &V = views[s];
      McState &m = mc[s];
      if (!m.started && V.randm_started) { m.started = true; m.irand = V.randm_state; }
      CUDA_TRY(cudaMemcpyAsync(mc_x + S.aoff, P.x + S.aoff, sizeof(double4) * S.natom, cudaMemcpyDeviceToDevice, stream));
      if (S.use_lrf)
        CUDA_TRY(cudaMemcpyAsync(mc_lrf + (size_t)S.coff * LRF_STRIDE, P.lrf + (size_t)S.coff * LRF_STRIDE,
                                 sizeof(double) * S.ncgp * LRF_STRIDE, cudaMemcpyDeviceToDevice, stream));
      SysState &t = st[s];
      const double old_V = t.boxl[0] * t.boxl[1] * t.boxl[2];
      double r = randm(m, V.pressure_seed);
      r = r * 2 - 1;
      const double deltaV = r * V.max_vol_displ, new_V = deltaV + old_V;
      const double ratio = std::pow(new_V / old_V, (double)(1.0f / 3.0f));
      for (int k = 0; k < 3; k++) {
        t.mc_oldl[k] = t.boxl[k];
        t.boxl[k] = t.boxl[k] * ratio;
        t.iboxl[k] = 1.0 / t.boxl[k];
      }
      const double bmin = std::min(t.boxl[0], std::min(t.boxl[1], t.boxl[2]));
      const char *why = !(bmin > V.Rcpp * 2)    ? "Solute-solute cut-off radii too large"
                        : !(bmin > V.Rcww * 2)  ? "Solvent-solvent cut-off radii too large"
                        : !(bmin > V.Rcpw * 2)  ? "Solute-solvent cut-off radii too large"
                        : !(bmin > V.Rcq * 2)   ? "Q-atom cut-off radii too large"
                        : !(bmin > V.RcLRF * 2) ? "LRF cut-off radii too large"
                                                : nullptr;
      if (why) {
        char buf[200];
        std::snprintf(buf, sizeof buf, "system %d, volume move after step %lld: %s", s, done, why);
        fail(QB_ERR_STATE, buf);
      }
      t.mc = 1;
      dV[s] = deltaV;
      oldV[s] = old_V;
      put_box(s, t);
    }
    CUDA_TRY(cudaStreamSynchronize(stream));   // st (host) is the source of the copies above
    launch("mc_scale", [&] { k_mc_scale<<<dim3(cdiv(max_nmol, 128), nsys), 128, 0, stream>>>(P); });
    bool lrf_any = false;
    for (int s : live) lrf_any |= sysh[s].use_lrf != 0;
    if (lrf_any) build_lists(2);
    // second new_potential: the trial box
    evaluate_into(E2, EQ2);
    std::vector<double> Efin = E0, EQfin = EQ0;
    for (int s : live) {
      const qb_sysview &V = views[s];
      McState &m = mc[s];
      const double *e0 = &E0[(size_t)s * QB_NE];
      const double p1 = new_potential(e0, &E1[(size_t)s * QB_NE]), p2 = new_potential(e0, &E2[(size_t)s * QB_NE]);
      SysState &t = st[s];
      const double newV = oldV[s] + dV[s];
      const double deltaE = p2 - p1;
      const double deltaW = deltaE + V.pressure * dV[s] -
                            (double)((float)V.nmol * kBoltz) * V.Temp0 * std::log(newV / oldV[s]);
      bool acc = true;
      if (deltaW > 0.0) {
        const double u = randm(m, V.pressure_seed);
        acc = !(u > std::exp(-deltaW / (double)kBoltz / V.Temp0));
      }
      m.tries++;
      if (acc) m.accepted++;
      const std::vector<double> &Es = acc ? E2 : E1, &EQs = acc ? EQ2 : EQ1;
      const double pot = acc ? p2 : p1;
      // the fields new_potential writes (md.f90:15858-15971)
      double *ef = &Efin[(size_t)s * QB_NE];
      const double *es = &Es[(size_t)s * QB_NE];
      for (int k : {QB_E_PP_EL, QB_E_PP_VDW, QB_E_PW_EL, QB_E_PW_VDW, QB_E_WW_EL, QB_E_WW_VDW, QB_E_QX_EL, QB_E_QX_VDW,
                    QB_E_RST_PROTEIN, QB_E_LRF})
        ef[k] = es[k];
      ef[QB_E_POTENTIAL] = pot;
      for (int q = 0; q < V.nstates; q++) {
        double *qf = &EQfin[((size_t)s * MAXS + q) * QB_NEQ];
        const double *qs = &EQs[((size_t)s * MAXS + q) * QB_NEQ];
        for (int k : {QB_EQ_QQ_EL, QB_EQ_QQ_VDW, QB_EQ_QP_EL, QB_EQ_QP_VDW, QB_EQ_QW_EL, QB_EQ_QW_VDW, QB_EQ_QX_EL,
                      QB_EQ_QX_VDW, QB_EQ_RESTRAINT})
          qf[k] = qs[k];
      }
      const SysDev &S = sysh[s];
      if (!acc) {
        CUDA_TRY(cudaMemcpyAsync(P.x + S.aoff, mc_x + S.aoff, sizeof(double4) * S.natom, cudaMemcpyDeviceToDevice, stream));
        if (S.use_lrf)
          CUDA_TRY(cudaMemcpyAsync(P.lrf + (size_t)S.coff * LRF_STRIDE, mc_lrf + (size_t)S.coff * LRF_STRIDE,
                                   sizeof(double) * S.ncgp * LRF_STRIDE, cudaMemcpyDeviceToDevice, stream));
        for (int k = 0; k < 3; k++) { t.boxl[k] = t.mc_oldl[k]; t.iboxl[k] = 1.0 / t.boxl[k]; }
      }
      t.mc = 0;
      put_box(s, t);
      // the step's records take the final energies
      for (int kind = 0; kind < 2; kind++) {
        const int cyc = kind == 0 ? V.iout_cycle : V.iene_cycle;
        if (cyc <= 0 || done % cyc != 0 || (kind == 1 && done == 0)) continue;
        const int c = t.hist_n[kind] - 1;
        if (c < 0 || c >= P.hist_cap) continue;
        double *r = P.hist + (((size_t)kind * nsys + s) * P.hist_cap + c) * HIST_REC;
        CUDA_TRY(cudaMemcpyAsync(r + 1, ef, sizeof(double) * QB_NE, cudaMemcpyHostToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(r + 1 + QB_NE, &EQfin[(size_t)s * MAXS * QB_NEQ], sizeof(double) * MAXS * QB_NEQ,
                                 cudaMemcpyHostToDevice, stream));
      }
    }
    // every system's E and EQ as the step (and the moves) left them
    CUDA_TRY(cudaMemcpyAsync(P.E, Efin.data(), sizeof(double) * Efin.size(), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaMemcpyAsync(P.EQ, EQfin.data(), sizeof(double) * EQfin.size(), cudaMemcpyHostToDevice, stream));
    CUDA_TRY(cudaStreamSynchronize(stream));   // the host vectors are the copies' sources
  }
  double4 *mc_x = nullptr;
  double *mc_lrf = nullptr;
  double *xyz = nullptr;   // packed x, y, z of every atom (the batched host copies)
  int max_nmol = 0;

  // the box fields of system s's device state (edge lengths, inverses,
  // centre, volume-move flag and old lengths), leaving the rest as the
  // device has it
  void put_box(int s, const SysState &t) {
    const size_t off = offsetof(SysState, boxl), len = sizeof(SysState) - off;
    CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char *>(P.st + s) + off, reinterpret_cast<const char *>(&t) + off, len,
                             cudaMemcpyHostToDevice, stream));
  }

  // The kernels of one MD step (md_run's loop body, md.f90:4003-4175).
  void step_kernels(int due, int ene) {
    DevPtrs &p = P;
    if (due) build_lists(0, true);
    pot_energy(ene);
    // 3-constraint molecules (waters) take leapfrog and SHAKE in one pass; the
    // other atoms leapfrog, then the general SHAKE; the two paths move
    // disjoint atoms
    const bool fused = any_shake && p.nsh3 > 0;
    if (fused) fork_streams();
    if (fused)
      launch("leapfrog_shake3", [&] { k_leapfrog_shake3<<<cdiv(p.nsh3, 128), 128, 0, stream>>>(p); });
    cudaStream_t sl = fused && forking() ? side[0] : stream;
    if (p.n_lf > 0) launch("leapfrog", [&] { k_leapfrog<<<cdiv(p.n_lf, 256), 256, 0, sl>>>(p); });
    if (any_shake && p.nshg > 0)
      launch("shake_general", [&] { k_shake_general<<<p.nshg, SHG_BLOCK, p.shg_smem, sl>>>(p); });
    if (fused) join_streams();
    launch("finish", [&] { k_finish<<<nsys, 32, 0, stream>>>(p, 1); });
    check_launch("step kernels");
  }

  void sync_status() {
    CUDA_TRY(cudaStreamSynchronize(stream));
    std::vector<SysState> st(nsys);
    CUDA_TRY(cudaMemcpy(st.data(), P.st, sizeof(SysState) * nsys, cudaMemcpyDeviceToHost));
    for (int s = 0; s < nsys; s++)
      if (st[s].status != 0) {
        char buf[160];
        std::snprintf(buf, sizeof buf, "system %d raised status %d on the device at step %d", s, st[s].status,
                      st[s].istep);
        fail(st[s].status, buf);
      }
  }
};

// ------------------------------------------------------------- packing

namespace {


// The water-water force kernels' blocks: wpb consecutive waters of one
// system each, system by system, into the tile buffer (sized at build for 32
// waters per block).
void set_ww_tiles(Batch &B, int wpb) {
  std::vector<int2> tiles;
  for (int s = 0; s < B.nsys; s++)
    for (int i0 = 0; i0 < B.sysh[s].nwat; i0 += wpb) tiles.push_back(make_int2(s, i0));
  if (tiles.empty()) tiles.push_back(make_int2(0, 0));
  if ((long long)tiles.size() > B.ww_tiles_cap) fail(QB_ERR_ARG, "ww_waters_per_block below the tile buffer's size");
  CUDA_TRY(cudaMemcpy(B.P.ww_tiles, tiles.data(), tiles.size() * sizeof(int2), cudaMemcpyHostToDevice));
  B.P.n_ww_tiles = (int)tiles.size();
  B.ww_wpb = wpb;
}

void build(Batch &B, qb_handle *const *hs, int n) {
  B.nsys = n;
  B.views.resize(n);
  for (int s = 0; s < n; s++) {
    B.systems.push_back(&hs[s]->sys);
    hs[s]->sys.fill_view(&B.views[s]);
  }
  B.NB = B.views[0].NBcycle;

  // host staging
  std::vector<double4> x, v, d0;
  std::vector<float> crg, winv;
  std::vector<double> mass, lja, ljb, xtop;
  std::vector<int> iac, iq, cgp, asys;
  std::vector<uint8_t> flags, ljcod;
  std::vector<uint32_t> lx, l14;
  std::vector<std::vector<int>> exl_at, l14_at;   // per global atom: distant exclusion / 1-4 partners
  std::vector<int> cg_first, cg_last, cg_sw, cg_atoms, cg_sys;
  std::vector<int2> lrft;
  std::vector<PwAtom> pwa;
  std::vector<int> pwg_off;
  std::vector<int> iqseq, qiac;
  std::vector<float> qcrg;
  std::vector<double> qavdw, qbvdw, sc, qq_el;
  std::vector<int8_t> qconn;
  std::vector<int4> qq;
  std::vector<int2> bij; std::vector<double2> bpar;
  std::vector<int4> aijk; std::vector<double2> apar, aub;
  std::vector<int4> tijkl; std::vector<float4> tpar;
  std::vector<int4> iijkl; std::vector<float2> ipar;
  std::vector<int2> qbij; std::vector<uint8_t> qb_on; std::vector<double4> qbpar;
  std::vector<int4> qaijk; std::vector<uint8_t> qa_on; std::vector<double2> qapar, qaub;
  std::vector<int4> qtijkl; std::vector<uint8_t> qt_on; std::vector<double4> qtpar;
  std::vector<int4> qiijkl; std::vector<uint8_t> qi_on; std::vector<double2> qipar;
  std::vector<int2> qa_cpl, qt_cpl, qi_cpl; std::vector<int8_t> qa_src, qa_src_ub, qt_src, qi_src;
  std::vector<int> sh_first, sh_n, sh_sys; std::vector<int2> sh_ij; std::vector<double> sh_d2;
  std::vector<int4> rs; std::vector<double> rs_fk;
  std::vector<int2> rp; std::vector<double> rp_x, rp_fk;
  std::vector<int4> rd; std::vector<double4> rd_p;
  std::vector<int4> ra; std::vector<double2> ra_p;
  std::vector<int4> rw; std::vector<double4> rw_p;
  std::vector<int> mol_first; std::vector<double> mol_minv, mass_box;
  std::vector<SysState> sst(n);
  B.sysh.resize(n);
  int ww_cap = 64;
  long long pp_tot = 0, qp_tot = 0, qw_tot = 0;
  int ncgp_sol_tot = 0, pwg_cap = 32;

  for (int s = 0; s < n; s++) {
    const qb_sysview &V = B.views[s];
    SysDev &S = B.sysh[s];
    std::memset(&S, 0, sizeof S);
    if (V.nstates > MAXS) fail(QB_ERR_UNSUPPORTED, "too many states");

    const int aoff = (int)x.size();
    S.aoff = aoff; S.natom = V.natom; S.nsol = V.nat_solute; S.nwat = V.nwat;
    if (V.nwat > 65535) fail(QB_ERR_UNSUPPORTED, "more than 65535 waters in one system");
    S.woff = 0;
    S.coff = (int)cg_first.size(); S.ncgp = V.ncgp; S.ncgp_sol = V.ncgp_solute;
    S.qoff = (int)iqseq.size(); S.nq = V.nqat; S.S = V.nstates; S.natyps = V.natyps;
    S.ljoff = (int)ljcod.size(); S.qlib_off = (int)qavdw.size(); S.sc_off = (int)sc.size();
    S.qconn_off = (int)qconn.size();
    std::vector<char> shaken(V.natom, 0);
    for (int c = 0; c < V.shake_constraints; c++) shaken[V.shake_i[c]] = shaken[V.shake_j[c]] = 1;
    for (int i = 0; i < V.natom; i++) {
      x.push_back(make_double4(V.x0[3 * i], V.x0[3 * i + 1], V.x0[3 * i + 2], 0));
      v.push_back(make_double4(V.v0[3 * i], V.v0[3 * i + 1], V.v0[3 * i + 2], 0));
      for (int k = 0; k < 3; k++) xtop.push_back(V.xtop[3 * i + k]);
      crg.push_back(V.crg[i]);
      winv.push_back(V.winv[i]);
      mass.push_back(V.mass[i]);
      int t = V.iac[i];
      iac.push_back(t);
      for (int k = 0; k < 3; k++) { lja.push_back(V.type_avdw[3 * t + k]); ljb.push_back(V.type_bvdw[3 * t + k]); }
      iq.push_back(V.iqatom[i]);
      cgp.push_back(S.coff + V.iwhich_cgp[i]);
      asys.push_back(s);
      flags.push_back((V.excl[i] ? F_EXCL : 0) | (V.shell[i] ? F_SHELL : 0) | (V.heavy[i] ? F_HEAVY : 0) |
                      (shaken[i] ? F_SHAKE : 0));
      lx.push_back(i < V.nat_solute ? V.listex_bits[i] : 0u);
      l14.push_back(i < V.nat_solute ? V.list14_bits[i] : 0u);
    }
    for (int k = 0; k < V.natyps * V.natyps; k++) ljcod.push_back(V.ljcod[k]);
    exl_at.resize(x.size());
    l14_at.resize(x.size());
    for (int k = 0; k < V.nexlong; k++) {
      const int a = aoff + V.listexlong[2 * k], b = aoff + V.listexlong[2 * k + 1];
      exl_at[a].push_back(b);
      exl_at[b].push_back(a);
    }
    for (int k = 0; k < V.n14long; k++) {
      const int a = aoff + V.list14long[2 * k], b = aoff + V.list14long[2 * k + 1];
      l14_at[a].push_back(b);
      l14_at[b].push_back(a);
    }
    for (int g = 0; g < V.ncgp; g++) {
      cg_first.push_back((int)cg_atoms.size() + (V.cgp_first[g] - V.cgp_first[0]));
      cg_last.push_back((int)cg_atoms.size() + (V.cgp_last[g] - V.cgp_first[0]));
      cg_sw.push_back(aoff + V.cgp_iswitch[g]);
      cg_sys.push_back(s);
    }
    for (int a = 0; a < V.natom; a++) cg_atoms.push_back(aoff + V.cgpatom[a]);
    // LRF gather tiles: runs of consecutive groups with contiguous atom ranges
    S.lrft_off = (int)lrft.size(); S.nlrft = 0;
    if (V.use_LRF) {
      int h0 = 0;
      while (h0 < V.ncgp) {
        int h1 = h0 + 1;
        if (V.cgp_last[h0] - V.cgp_first[h0] + 1 > LRF_TILE_A)
          fail(QB_ERR_UNSUPPORTED, "a charge group has more atoms than the LRF tile holds");
        while (h1 < V.ncgp && h1 - h0 < LRF_TILE_G && V.cgp_first[h1] == V.cgp_last[h1 - 1] + 1 &&
               V.cgp_last[h1] - V.cgp_first[h0] + 1 <= LRF_TILE_A)
          h1++;
        lrft.push_back(make_int2(h0, h1));
        S.nlrft++;
        h0 = h1;
      }
    }
    // water groups must be O,H,H with the oxygen as switching atom
    for (int iw = 0; iw < V.nwat; iw++) {
      int g = V.ncgp_solute + iw;
      int o = V.nat_solute + 3 * iw;
      if (g >= V.ncgp || V.cgp_iswitch[g] != o || V.iwhich_cgp[o] != g)
        fail(QB_ERR_UNSUPPORTED, "water charge groups must follow the solute groups, one per water, switching on O");
      // one water model: the solute-water kernel takes charges and types from the first water
      const int o0 = V.nat_solute;
      for (int k = 0; k < 3; k++)
        if (V.crg[o + k] != V.crg[o0 + (k ? 1 : 0)] || V.iac[o + k] != V.iac[o0 + (k ? 1 : 0)])
          fail(QB_ERR_UNSUPPORTED, "waters must share one charge and atom type per site (O, H, H)");
    }
    // Q atoms
    for (int q = 0; q < V.nqat; q++) {
      iqseq.push_back(aoff + V.iqseq[q]);
      for (int st = 0; st < MAXS; st++) {
        qcrg.push_back(st < V.nstates ? V.qcrg[q * V.nstates + st] : 0.0f);
        qiac.push_back(st < V.nstates ? V.qiac[q * V.nstates + st] : 0);
      }
    }
    for (int k = 0; k < V.nqlib * 3; k++) { qavdw.push_back(V.qavdw[k]); qbvdw.push_back(V.qbvdw[k]); }
    size_t nsc = (size_t)V.nqat * (V.natyps + V.nqat) * V.nstates;
    for (size_t k = 0; k < nsc; k++) sc.push_back(V.sc_lookup[k]);
    size_t nqc = (size_t)V.nstates * V.nat_solute * V.nqat;
    for (size_t k = 0; k < nqc; k++) qconn.push_back(V.qconn[k]);
    S.qq_off = (int)qq.size();
    for (int st = 0; st < V.nstates; st++)
      for (int k = V.nbqq_off[st]; k < V.nbqq_off[st] + V.nbqq_count[st]; k++) {
        int jq = V.nbqq_jq[k];
        qq.push_back(make_int4(S.qoff + V.nbqq_iq[k], aoff + V.nbqq_j[k], jq >= 0 ? S.qoff + jq : -1,
                               V.nbqq_ljcod[k] | (st << 8)));
        qq_el.push_back(V.nbqq_el_scale[k]);
      }
    S.nqq = (int)qq.size() - S.qq_off;
    // bonded terms
    S.b_off = (int)bij.size(); S.nb = V.nbonds; S.nb_sol = V.nbonds_solute;
    for (int k = 0; k < V.nbonds; k++) {
      bij.push_back(make_int2(aoff + V.bnd_i[k], aoff + V.bnd_j[k]));
      bpar.push_back(make_double2(V.bnd_fk[k], V.bnd_b0[k]));
    }
    S.a_off = (int)aijk.size(); S.na = V.nangles; S.na_sol = V.nangles_solute;
    for (int k = 0; k < V.nangles; k++) {
      aijk.push_back(make_int4(aoff + V.ang_i[k], aoff + V.ang_j[k], aoff + V.ang_k[k], 0));
      apar.push_back(make_double2(V.ang_fk[k], V.ang_th0[k]));
      aub.push_back(make_double2(V.ang_ureyfk[k], V.ang_ureyr0[k]));
    }
    S.t_off = (int)tijkl.size(); S.nt = V.ntors; S.nt_sol = V.ntors_solute;
    for (int k = 0; k < V.ntors; k++) {
      tijkl.push_back(make_int4(aoff + V.tor_i[k], aoff + V.tor_j[k], aoff + V.tor_k[k], aoff + V.tor_l[k]));
      tpar.push_back(make_float4(V.tor_fk[k], V.tor_rmult[k], V.tor_deltor[k], V.tor_paths[k]));
    }
    S.i_off = (int)iijkl.size(); S.ni = V.nimps; S.ni_sol = V.nimps_solute;
    for (int k = 0; k < V.nimps; k++) {
      iijkl.push_back(make_int4(aoff + V.imp_i[k], aoff + V.imp_j[k], aoff + V.imp_k[k], aoff + V.imp_l[k]));
      ipar.push_back(make_float2(V.imp_fk[k], V.imp_imp0[k]));
    }
    const int NSt = V.nstates;
    S.qb_off = (int)qbij.size(); S.nqb = V.nqbond;
    for (int k = 0; k < V.nqbond; k++) {
      qbij.push_back(make_int2(aoff + V.qbnd_i[k], aoff + V.qbnd_j[k]));
      for (int st = 0; st < MAXS; st++) {
        bool on = st < NSt && V.qbnd_on[k * NSt + st];
        qb_on.push_back(on);
        qbpar.push_back(on ? make_double4(V.qbnd_Dmz[k * NSt + st], V.qbnd_amz[k * NSt + st], V.qbnd_r0[k * NSt + st],
                                          V.qbnd_fk[k * NSt + st])
                           : make_double4(0, 0, 0, 0));
      }
    }
    S.qa_off = (int)qaijk.size(); S.nqa = V.nqangle;
    for (int k = 0; k < V.nqangle; k++) {
      qaijk.push_back(make_int4(aoff + V.qang_i[k], aoff + V.qang_j[k], aoff + V.qang_k[k], 0));
      for (int st = 0; st < MAXS; st++) {
        bool on = st < NSt && V.qang_on[k * NSt + st];
        qa_on.push_back(on);
        qapar.push_back(on ? make_double2(V.qang_fk[k * NSt + st], V.qang_th0[k * NSt + st]) : make_double2(0, 0));
        qaub.push_back(on ? make_double2(V.qang_ureyfk[k * NSt + st], V.qang_ureyr0[k * NSt + st]) : make_double2(0, 0));
        qa_src.push_back((int8_t)(st < NSt ? V.qang_cpl_src[k * NSt + st] : -1));
        qa_src_ub.push_back((int8_t)(st < NSt ? V.qang_cpl_ub_src[k * NSt + st] : -1));
      }
      qa_cpl.push_back(make_int2(V.qang_cpl[k] >= 0 ? S.qb_off + V.qang_cpl[k] : -1,
                                 V.qang_cpl_ub[k] >= 0 ? S.qb_off + V.qang_cpl_ub[k] : -1));
    }
    S.qt_off = (int)qtijkl.size(); S.nqt = V.nqtor;
    for (int k = 0; k < V.nqtor; k++) {
      qtijkl.push_back(make_int4(aoff + V.qtor_i[k], aoff + V.qtor_j[k], aoff + V.qtor_k[k], aoff + V.qtor_l[k]));
      for (int st = 0; st < MAXS; st++) {
        bool on = st < NSt && V.qtor_on[k * NSt + st];
        qt_on.push_back(on);
        qtpar.push_back(on ? make_double4(V.qtor_fk[k * NSt + st], V.qtor_rmult[k * NSt + st], V.qtor_deltor[k * NSt + st], 0)
                           : make_double4(0, 0, 0, 0));
        qt_src.push_back((int8_t)(st < NSt ? V.qtor_cpl_src[k * NSt + st] : -1));
      }
      qt_cpl.push_back(make_int2(V.qtor_cpl[k] >= 0 ? S.qb_off + V.qtor_cpl[k] : -1, 0));
    }
    S.qi_off = (int)qiijkl.size(); S.nqi = V.nqimp;
    for (int k = 0; k < V.nqimp; k++) {
      qiijkl.push_back(make_int4(aoff + V.qimp_i[k], aoff + V.qimp_j[k], aoff + V.qimp_k[k], aoff + V.qimp_l[k]));
      for (int st = 0; st < MAXS; st++) {
        bool on = st < NSt && V.qimp_on[k * NSt + st];
        qi_on.push_back(on);
        qipar.push_back(on ? make_double2(V.qimp_fk[k * NSt + st], V.qimp_imp0[k * NSt + st]) : make_double2(0, 0));
        qi_src.push_back((int8_t)(st < NSt ? V.qimp_cpl_src[k * NSt + st] : -1));
      }
      qi_cpl.push_back(make_int2(V.qimp_cpl[k] >= 0 ? S.qb_off + V.qimp_cpl[k] : -1, V.qimp_cpl_flag[k]));
    }
    S.noffd = V.noffd;
    if (S.noffd > MAXS) fail(QB_ERR_ARG, "too many off-diagonal functions");
    for (int k = 0; k < V.noffd; k++) {
      S.offd_k[k] = aoff + V.iqseq[V.offd_k[k]];
      S.offd_l[k] = aoff + V.iqseq[V.offd_l[k]];
    }
    // shake molecules
    S.sh_off = (int)sh_first.size(); S.nsh = V.shake_molecules;
    for (int m = 0; m < V.shake_molecules; m++) {
      sh_first.push_back((int)sh_ij.size() + (V.shake_mol_first[m] - (V.shake_molecules ? V.shake_mol_first[0] : 0)));
      sh_n.push_back(V.shake_mol_n[m]);
      sh_sys.push_back(s);
    }
    for (int c = 0; c < V.shake_constraints; c++) {
      sh_ij.push_back(make_int2(aoff + V.shake_i[c], aoff + V.shake_j[c]));
      sh_d2.push_back(V.shake_dist2[c]);
    }
    S.has_shake = V.shake_constraints > 0;
    // restraints
    S.rs_off = (int)rs.size(); S.nrs = V.nrstr_seq;
    for (int r = 0; r < V.nrstr_seq; r++) {
      rs.push_back(make_int4(aoff + V.rseq_i[r], aoff + V.rseq_j[r], V.rseq_ih[r], V.rseq_to_center[r]));
      rs_fk.push_back(V.rseq_fk[r]);
    }
    S.rp_off = (int)rp.size(); S.nrp = V.nrstr_pos;
    for (int r = 0; r < V.nrstr_pos; r++) {
      rp.push_back(make_int2(aoff + V.rpos_i[r], V.rpos_ipsi[r]));
      for (int k = 0; k < 3; k++) { rp_x.push_back(V.rpos_x[3 * r + k]); rp_fk.push_back(V.rpos_fk[3 * r + k]); }
    }
    S.rd_off = (int)rd.size(); S.nrd = V.nrstr_dist;
    for (int r = 0; r < V.nrstr_dist; r++) {
      rd.push_back(make_int4(aoff + V.rdis_i[r], aoff + V.rdis_j[r], V.rdis_ipsi[r], 0));
      rd_p.push_back(make_double4(V.rdis_d1[r], V.rdis_d2[r], V.rdis_fk[r], 0));
    }
    S.ra_off = (int)ra.size(); S.nra = V.nrstr_angl;
    for (int r = 0; r < V.nrstr_angl; r++) {
      ra.push_back(make_int4(aoff + V.rang_i[r], aoff + V.rang_j[r], aoff + V.rang_k[r], V.rang_ipsi[r]));
      ra_p.push_back(make_double2(V.rang_ang[r], V.rang_fk[r]));
    }
    S.rw_off = (int)rw.size(); S.nrw = V.nrstr_wall;
    for (int r = 0; r < V.nrstr_wall; r++) {
      rw.push_back(make_int4(aoff + V.rwal_i[r], aoff + V.rwal_j[r], V.rwal_ih[r], 0));
      rw_p.push_back(make_double4(V.rwal_d[r], V.rwal_fk[r], V.rwal_aMorse[r], V.rwal_dMorse[r]));
    }
    // scalars
    S.switch_atoms = V.iuse_switch_atom == 1 ? 1 : 0;
    if (!S.switch_atoms) B.any_any_atom = true;
    S.ff_type = V.ff_type; S.use_lrf = V.use_LRF; S.qvdw = V.qvdw_flag; S.qq_lib = V.qq_use_library_charges;
    S.wpol = V.wpol_restr && V.nwpolr_shell > 0; S.nshell = V.nwpolr_shell;
    if (S.wpol) B.max_nshell = std::max(B.max_nshell, std::min(S.nshell, MAX_SHELLS));
    if (S.nshell > MAX_SHELLS) fail(QB_ERR_UNSUPPORTED, "too many water polarisation shells");
    S.iac_ow = V.iac_ow; S.separate_scaling = V.separate_scaling; S.detail_temps = V.detail_temps;
    S.qp_once = V.Rcq > V.rexcl_o;
    S.iout = V.iout_cycle; S.iene = V.iene_cycle; S.NB = V.NBcycle;
    S.Ndegf = V.Ndegf; S.Ndegfree = V.Ndegfree; S.Ndegfree_sol = V.Ndegfree_solute; S.Ndegfree_solv = V.Ndegfree_solvent;
    S.dt = V.dt; S.Temp0 = V.Temp0; S.tau_T = V.tau_T; S.el14 = V.el14_scale; S.A_OO = V.A_OO; S.B_OO = V.B_OO;
    S.Rcpp2 = V.Rcpp * V.Rcpp; S.Rcpw2 = V.Rcpw * V.Rcpw; S.Rcww2 = V.Rcww * V.Rcww; S.Rcq2 = V.Rcq * V.Rcq;
    S.RcLRF2 = V.RcLRF * V.RcLRF;
    S.crg_ow = V.crg_ow; S.crg_hw = V.crg_hw;
    for (int k = 0; k < 3; k++) { S.xp[k] = V.xpcent[k]; S.xw[k] = V.xwcent[k]; }
    S.rwat = V.rwat; S.fk_ws = V.fk_wsphere; S.Dwmz = V.Dwmz; S.awmz = V.awmz; S.fkwpol = V.fkwpol;
    S.fk_pshell = V.fk_pshell; S.fk_fix = V.fk_fix;
    for (int k = 0; k < S.nshell; k++) { S.ws_rout[k] = V.wshell_rout[k]; S.ws_dr[k] = V.wshell_dr[k]; S.ws_cstb[k] = V.wshell_cstb[k]; }
    for (int k = 0; k < V.nstates; k++) S.lambda[k] = V.lambda[k];
    S.arith = V.ivdw_rule == 2 ? 1 : 0;
    if (V.nwat > 0) {
      S.aO[0] = V.type_avdw[3 * V.iac_ow]; S.aO[1] = V.type_avdw[3 * V.iac_ow + 1];
      S.bO[0] = V.type_bvdw[3 * V.iac_ow]; S.bO[1] = V.type_bvdw[3 * V.iac_ow + 1];
      S.hlj = V.ww_hlj; S.iac_hw = V.iac_hw;
      S.A_OH = V.A_OH; S.B_OH = V.B_OH; S.A_HH = V.A_HH; S.B_HH = V.B_HH;
      S.aH[0] = V.type_avdw[3 * V.iac_hw]; S.aH[1] = V.type_avdw[3 * V.iac_hw + 1];
      S.bH[0] = V.type_bvdw[3 * V.iac_hw]; S.bH[1] = V.type_bvdw[3 * V.iac_hw + 1];
    }
    SysState &st = sst[s];
    std::memset(&st, 0, sizeof st);
    st.Tscale_sol = st.Tscale_solv = 1.0;
    for (int k = 0; k < S.nshell; k++) st.theta_corr[k] = V.wshell_theta_corr0[k];
    // periodic box (use_PBC, md.f90:4000-4200): box, Q switching atom and
    // molecule tables; any-atom cut-offs stay sphere-only here
    S.pbc = V.use_pbc ? 1 : 0;
    for (int k = 0; k < 3; k++) S.origin[k] = V.xpcent[k];
    if (S.pbc) {
      if (V.iuse_switch_atom != 1)
        fail(QB_ERR_UNSUPPORTED, "any-atom charge-group cut-offs (iuse_switch_atom 0) in a periodic box are not supported");
      if (V.nqat > 0 && V.qswitch < 0) fail(QB_ERR_PARSE, "a periodic box needs the Q atoms' switching atom");
      S.qswitch = V.qswitch >= 0 ? aoff + V.qswitch : aoff;
      S.qp_once = 0;
      S.rigid_center = V.rigid_box_center;
      for (int k = 0; k < 3; k++) {
        sst[s].boxl[k] = V.boxlength[k];
        sst[s].iboxl[k] = 1.0 / V.boxlength[k];
        sst[s].boxc[k] = V.boxcenter[k];
        S.origin[k] = V.boxcenter[k];
      }
      S.mol_off = (int)mol_first.size();
      S.nmol = V.nmol;
      // both tables take nmol + 1 entries per system (one offset for both)
      for (int m = 0; m <= V.nmol; m++) mol_first.push_back(aoff + V.istart_mol[m]);
      for (int m = 0; m <= V.nmol; m++) mol_minv.push_back(m < V.nmol ? V.mol_mass_inv[m] : 0.0);
      // put_back_in_box's molecule range (md.f90:15529-15536): the solvent
      // molecules are the last (natom - nat_solute) / (atoms of the last one)
      S.put_first = 0; S.put_last = 0;
      if ((V.put_solute_back_in_box || V.put_solvent_back_in_box) && V.nmol > 1) {
        const int nsolv = (V.natom - V.nat_solute) / (V.istart_mol[V.nmol - 1] - V.istart_mol[V.nmol - 2]);
        S.put_first = V.put_solute_back_in_box ? 0 : V.nmol - nsolv;
        S.put_last = V.put_solvent_back_in_box ? V.nmol : V.nmol - nsolv;
        if (S.put_first < S.put_last) B.any_put = true;
      }
      B.any_box = true;
      if (V.constant_pressure) B.any_npt = true;
    }
    for (int i = 0; i < V.natom; i++) mass_box.push_back(S.pbc ? V.mass_box[i] : V.mass[i]);
    // list capacities from the starting coordinates, with margins for motion
    // (distances of the nearest image in a periodic box)
    {
      const double *X = V.x0;
      const bool pb = S.pbc != 0;
      auto d2 = [&](const double *x, int a, int b) {
        double t = 0;
        for (int k = 0; k < 3; k++) {
          double d = x[3 * a + k] - x[3 * b + k];
          if (pb) d -= V.boxlength[k] * std::round(d / V.boxlength[k]);
          t += d * d;
        }
        return t;
      };
      long long pp = 0;
      int pwmax = 0;
      double rpp = V.Rcpp + 3.0, rpw = V.Rcpw + 3.0, rww = V.Rcww + 2.0;
      for (int ig = 0; ig < V.ncgp_solute; ig++) {
        int si = V.cgp_iswitch[ig];
        int na = V.cgp_last[ig] - V.cgp_first[ig] + 1;
        for (int jg = ig; jg < V.ncgp_solute; jg++) {
          int sj = V.cgp_iswitch[jg];
          if (d2(X, si, sj) <= rpp * rpp) pp += (long long)na * (V.cgp_last[jg] - V.cgp_first[jg] + 1);
        }
        int c = 0;
        for (int iw = 0; iw < V.nwat; iw++)
          if (d2(X, si, V.nat_solute + 3 * iw) <= rpw * rpw) c++;
        pwmax = std::max(pwmax, c);
      }
      S.pp_cap = (int)(pp * 1.3 + 256);
      if (V.nwat > 0 && V.ncgp_solute > 0)
        pwg_cap = std::max(pwg_cap, std::min(((int)(pwmax * 1.15) + 32 + 31) / 32 * 32, (V.nwat + 31) / 32 * 32));
      S.qp_cap = V.nqat * V.nat_solute + 16;
      S.qw_cap = V.nwat + 16;
      int mx = 0;
      for (int iw = 0; iw < V.nwat; iw++) {
        int c = 0;
        for (int jw = 0; jw < V.nwat; jw++)
          if (jw != iw && d2(X, V.nat_solute + 3 * iw, V.nat_solute + 3 * jw) <= rww * rww) c++;
        mx = std::max(mx, c);
      }
      ww_cap = std::max(ww_cap, ((int)(mx * 1.15) + 31) / 32 * 32);
    }
    S.pp_off = (int)pp_tot; pp_tot += S.pp_cap;
    S.csoff = ncgp_sol_tot; ncgp_sol_tot += V.ncgp_solute;
    // solute-water tables: each solute group's non-Q atoms with their charge
    // products (single precision, as crg(i)*crg(j)) and LJ products with the
    // water O and H types
    for (int ig = 0; ig < V.ncgp_solute; ig++) {
      pwg_off.push_back((int)pwa.size());
      if (V.nwat == 0) continue;
      const int o = V.nat_solute;            // first water O; H is o + 1
      const int to = V.iac[o], th = V.iac[o + 1];
      for (int a = V.cgp_first[ig]; a <= V.cgp_last[ig]; a++) {
        const int i = V.cgpatom[a];
        if (V.iqatom[i] >= 0) continue;
        const int ti = V.iac[i];
        const int lo = V.ljcod[ti * V.natyps + to], lh = V.ljcod[ti * V.natyps + th];
        PwAtom r;
        double Ao, Bo, Ah, Bh;
        lj_pair(V.ivdw_rule == 2, V.type_avdw[3 * ti + lo - 1], V.type_avdw[3 * to + lo - 1],
                V.type_bvdw[3 * ti + lo - 1], V.type_bvdw[3 * to + lo - 1], Ao, Bo);
        lj_pair(V.ivdw_rule == 2, V.type_avdw[3 * ti + lh - 1], V.type_avdw[3 * th + lh - 1],
                V.type_bvdw[3 * ti + lh - 1], V.type_bvdw[3 * th + lh - 1], Ah, Bh);
        r.lj = make_double4(Ao, Bo, Ah, Bh);
        r.q = make_float2(V.crg[i] * V.crg[o], V.crg[i] * V.crg[o + 1]);
        r.atom = aoff + i;
        r.pad = 0;
        pwa.push_back(r);
      }
    }
    S.qp_off = (int)qp_tot; qp_tot += S.qp_cap;
    S.qw_off = (int)qw_tot; qw_tot += S.qw_cap;
    B.max_natom = std::max(B.max_natom, V.natom);
    B.max_nsol = std::max(B.max_nsol, V.nat_solute);
    B.max_nwat = std::max(B.max_nwat, V.nwat);
    B.max_ncgp_sol = std::max(B.max_ncgp_sol, V.ncgp_solute);
    B.max_ncgp = std::max(B.max_ncgp, V.ncgp);
    if (V.use_LRF) B.lrf_dims.push_back(make_int2(V.ncgp, S.nlrft));
    B.max_terms = std::max(B.max_terms, V.nbonds + V.nangles + V.ntors + V.nimps);
    B.max_pp = std::max(B.max_pp, S.pp_cap);
    if (V.nwat > 0) B.max_ncgp_sol_w = std::max(B.max_ncgp_sol_w, V.ncgp_solute);
    B.max_qp = std::max(B.max_qp, S.qp_cap);
    B.any_lrf |= V.use_LRF != 0;
    if (V.nqat > 0) B.q_states = (!B.any_q || B.q_states == V.nstates) ? V.nstates : 0;
    B.any_q |= V.nqat > 0;
    B.max_nq = std::max(B.max_nq, V.nqat);
    B.any_shake |= V.shake_constraints > 0;
    B.any_wpol |= S.wpol != 0;
    B.any_prestr |= (V.nrstr_seq + V.nrstr_pos + V.nrstr_dist + V.nrstr_angl + V.nrstr_wall) > 0;
    B.any_qq |= S.nqq > 0;
    B.any_qb |= (V.nqbond + V.nqangle + V.nqtor + V.nqimp + V.noffd) > 0;   // the Q-bonded block also takes r_kl
    B.any_hlj |= V.nwat > 0 && V.ww_hlj;
    if (S.pbc) B.max_nmol = std::max(B.max_nmol, V.nmol);
  }
  B.mc.assign(n, Batch::McState{});
  // water offsets
  int woff = 0;
  for (int s = 0; s < n; s++) { B.sysh[s].woff = woff; woff += B.sysh[s].nwat; }

  // device upload
  DevPtrs &P = B.P;
  P.nsys = n;
  P.natoms_tot = (int)x.size();
  P.nwat_tot = woff;
  P.ncgp_tot = (int)cg_first.size();
  P.nshake_tot = (int)sh_first.size();
  auto &o = B.owned;
  P.sys = dev_upload(B.sysh, o);
  P.st = dev_upload(sst, o);
  P.x = dev_upload(x, o); P.v = dev_upload(v, o);
  P.xx = dev_alloc<double4>(x.size(), o); P.d = dev_alloc<double4>(x.size(), o);
  P.crg = dev_upload(crg, o); P.winv = dev_upload(winv, o); P.mass = dev_upload(mass, o);
  P.iac = dev_upload(iac, o); P.iq = dev_upload(iq, o); P.cgp = dev_upload(cgp, o); P.asys = dev_upload(asys, o);
  P.flags = dev_upload(flags, o); P.lja = dev_upload(lja, o); P.ljb = dev_upload(ljb, o);
  P.lx = dev_upload(lx, o); P.l14 = dev_upload(l14, o);
  {
    auto csr = [&](const std::vector<std::vector<int>> &at, int *&off_d, int *&part_d) {
      std::vector<int> off(1, 0), part;
      for (size_t a = 0; a < x.size(); a++) {
        if (a < at.size()) part.insert(part.end(), at[a].begin(), at[a].end());
        off.push_back((int)part.size());
      }
      if (part.empty()) part.push_back(-1);
      off_d = dev_upload(off, o);
      part_d = dev_upload(part, o);
    };
    csr(exl_at, P.exo, P.exq);
    csr(l14_at, P.l14o, P.l14q);
  }
  P.ljcod = dev_upload(ljcod, o);
  P.xtop = dev_upload(xtop, o);
  P.cg_first = dev_upload(cg_first, o); P.cg_last = dev_upload(cg_last, o); P.cg_sw = dev_upload(cg_sw, o);
  P.cg_atoms = dev_upload(cg_atoms, o); P.cg_sys = dev_upload(cg_sys, o);
  P.lrf = dev_alloc<double>((size_t)P.ncgp_tot * LRF_STRIDE, o);
  P.lrft = dev_upload(lrft, o);
  P.iqseq = dev_upload(iqseq, o); P.qcrg = dev_upload(qcrg, o); P.qiac = dev_upload(qiac, o);
  P.qavdw = dev_upload(qavdw, o); P.qbvdw = dev_upload(qbvdw, o); P.sc = dev_upload(sc, o);
  P.qconn = dev_upload(qconn, o); P.qq = dev_upload(qq, o); P.qq_el = dev_upload(qq_el, o);
  P.bij = dev_upload(bij, o); P.bpar = dev_upload(bpar, o); P.aijk = dev_upload(aijk, o); P.apar = dev_upload(apar, o); P.aub = dev_upload(aub, o);
  P.tijkl = dev_upload(tijkl, o); P.tpar = dev_upload(tpar, o); P.iijkl = dev_upload(iijkl, o); P.ipar = dev_upload(ipar, o);
  P.qbij = dev_upload(qbij, o); P.qb_on = dev_upload(qb_on, o); P.qbpar = dev_upload(qbpar, o);
  P.qaijk = dev_upload(qaijk, o); P.qa_on = dev_upload(qa_on, o); P.qapar = dev_upload(qapar, o); P.qaub = dev_upload(qaub, o);
  P.qa_cpl = dev_upload(qa_cpl, o); P.qt_cpl = dev_upload(qt_cpl, o); P.qi_cpl = dev_upload(qi_cpl, o);
  P.qa_src = dev_upload(qa_src, o); P.qa_src_ub = dev_upload(qa_src_ub, o);
  P.qt_src = dev_upload(qt_src, o); P.qi_src = dev_upload(qi_src, o);
  P.qtijkl = dev_upload(qtijkl, o); P.qt_on = dev_upload(qt_on, o); P.qtpar = dev_upload(qtpar, o);
  P.qiijkl = dev_upload(qiijkl, o); P.qi_on = dev_upload(qi_on, o); P.qipar = dev_upload(qipar, o);
  P.sh_first = dev_upload(sh_first, o); P.sh_n = dev_upload(sh_n, o); P.sh_sys = dev_upload(sh_sys, o);
  P.sh_ij = dev_upload(sh_ij, o); P.sh_d2 = dev_upload(sh_d2, o);
  {
    // rigid three-site molecules: relabel atoms so the constraints, in order,
    // join (0,1), (0,2), (1,2)
    std::vector<int4> at3; std::vector<double4> d3; std::vector<int> gen;
    for (int m = 0; m < (int)sh_first.size(); m++) {
      int f = sh_first[m];
      bool tri = false;
      if (sh_n[m] == 3) {
        auto common = [](int2 a, int2 b) {
          if (a.x == b.x || a.x == b.y) return a.x;
          if (a.y == b.x || a.y == b.y) return a.y;
          return -1;
        };
        int2 c0 = sh_ij[f], c1 = sh_ij[f + 1], c2 = sh_ij[f + 2];
        int l0 = common(c0, c1), l1 = common(c0, c2), l2 = common(c1, c2);
        auto joins = [](int2 c, int a, int b) { return (c.x == a && c.y == b) || (c.x == b && c.y == a); };
        if (l0 >= 0 && l1 >= 0 && l2 >= 0 && l0 != l1 && l0 != l2 && l1 != l2 && joins(c0, l0, l1) &&
            joins(c1, l0, l2) && joins(c2, l1, l2)) {
          at3.push_back(make_int4(l0, l1, l2, sh_sys[m]));
          d3.push_back(make_double4(sh_d2[f], sh_d2[f + 1], sh_d2[f + 2], 0.0));
          tri = true;
        }
      }
      if (!tri) gen.push_back(m);
    }
    P.nsh3 = (int)at3.size(); P.nshg = (int)gen.size();
    P.sh3_at = dev_upload(at3, o); P.sh3_d2 = dev_upload(d3, o);
    // their atoms are moved by the fused leapfrog + SHAKE kernel, not k_leapfrog
    for (auto &a : at3) { flags[a.x] |= F_SH3; flags[a.y] |= F_SH3; flags[a.z] |= F_SH3; }
    if (!at3.empty()) CUDA_TRY(cudaMemcpy(P.flags, flags.data(), flags.size(), cudaMemcpyHostToDevice));
    {
      std::vector<int> lf;
      for (int g = 0; g < (int)flags.size(); g++)
        if (!(flags[g] & F_SH3)) lf.push_back(g);
      P.n_lf = (int)lf.size();
      P.lf_atoms = dev_upload(lf, o);
    }
    {
      std::vector<int2> pk, wp, qw;
      for (int s = 0; s < n; s++) {
        const SysDev &S = B.sysh[s];
        for (int i0 = 0; i0 < std::max(S.nwat, S.nsol); i0 += 256) pk.push_back(make_int2(s, i0));
        if (S.wpol && S.nshell > 0)
          for (int i0 = 0; i0 < S.nwat; i0 += WPOL_BLOCK) wp.push_back(make_int2(s, i0));
        if (S.nq > 0)
          for (int i0 = 0; i0 < S.nwat; i0 += 128) qw.push_back(make_int2(s, i0));
      }
      std::vector<int2> pwg;
      for (int s = 0; s < n; s++)
        if (B.sysh[s].nwat > 0)
          for (int ig = 0; ig < B.sysh[s].ncgp_sol; ig++) pwg.push_back(make_int2(s, ig));
      P.n_pw_groups = (int)pwg.size();
      P.pw_groups = dev_upload(pwg, o);
      P.n_pk_tiles = (int)pk.size(); P.n_wp_tiles = (int)wp.size(); P.n_qw_tiles = (int)qw.size();
      P.pk_tiles = dev_upload(pk, o); P.wp_tiles = dev_upload(wp, o); P.qw_tiles = dev_upload(qw, o);
    }
    // other molecules: local atoms, constraints grouped into dependency levels
    std::vector<int4> info, info2;
    std::vector<int> gat, glev;
    std::vector<int2> gc;
    std::vector<double> gd2;
    size_t smem_max = 0;
    long long scratch = 0;
    const size_t smem_cap = 200 * 1024;
    for (int m : gen) {
      int f = sh_first[m], n = sh_n[m];
      std::map<int, int> loc;
      std::vector<int> atoms;
      for (int c = 0; c < n; c++)
        for (int a : {sh_ij[f + c].x, sh_ij[f + c].y})
          if (!loc.count(a)) { loc[a] = (int)atoms.size(); atoms.push_back(a); }
      std::vector<int> last(atoms.size(), 0), level(n);
      int nlev = 0;
      for (int c = 0; c < n; c++) {
        int i = loc[sh_ij[f + c].x], j = loc[sh_ij[f + c].y];
        level[c] = std::max(last[i], last[j]) + 1;
        last[i] = last[j] = level[c];
        nlev = std::max(nlev, level[c]);
      }
      int4 in = make_int4((int)gat.size(), (int)atoms.size(), (int)gc.size(), n);
      gat.insert(gat.end(), atoms.begin(), atoms.end());
      int loff = (int)glev.size();
      for (int L = 1; L <= nlev; L++) {
        glev.push_back((int)gc.size() - in.z);
        for (int c = 0; c < n; c++)
          if (level[c] == L) {
            gc.push_back(make_int2(loc[sh_ij[f + c].x], loc[sh_ij[f + c].y]));
            gd2.push_back(sh_d2[f + c]);
          }
      }
      glev.push_back((int)gc.size() - in.z);
      size_t bytes = (size_t)(in.y + n) * sizeof(double4) + (size_t)n;
      int soff = -1;
      if (bytes <= smem_cap) smem_max = std::max(smem_max, bytes);
      else { soff = (int)scratch; scratch += in.y + n + (n + 31) / 32; }
      info.push_back(in);
      info2.push_back(make_int4(loff, nlev, sh_sys[m], soff));
    }
    P.shg_info = dev_upload(info, o); P.shg_info2 = dev_upload(info2, o);
    P.shg_at = dev_upload(gat, o); P.shg_c = dev_upload(gc, o); P.shg_d2 = dev_upload(gd2, o);
    P.shg_lev = dev_upload(glev, o);
    P.shg_scratch = dev_alloc<double4>((size_t)std::max<long long>(scratch, 1), o);
    P.shg_smem = (smem_max + 15) / 16 * 16;
    if (P.nshg > 0)
      CUDA_TRY(cudaFuncSetAttribute(k_shake_general, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
  }
  if (mol_first.empty()) mol_first.push_back(0);
  if (mol_minv.empty()) mol_minv.push_back(0.0);
  P.mol_first = dev_upload(mol_first, o); P.mol_minv = dev_upload(mol_minv, o); P.mass_box = dev_upload(mass_box, o);
  P.rs = dev_upload(rs, o); P.rs_fk = dev_upload(rs_fk, o); P.rp = dev_upload(rp, o); P.rp_x = dev_upload(rp_x, o);
  P.rp_fk = dev_upload(rp_fk, o); P.rd = dev_upload(rd, o); P.rd_p = dev_upload(rd_p, o);
  P.ra = dev_upload(ra, o); P.ra_p = dev_upload(ra_p, o); P.rw = dev_upload(rw, o); P.rw_p = dev_upload(rw_p, o);
  P.pp = dev_alloc<int4>(pp_tot, o);
  P.pwg_cap = pwg_cap;
  P.pwg = dev_alloc<uint16_t>((size_t)std::max(ncgp_sol_tot, 1) * pwg_cap, o);
  P.pwg_n = dev_alloc<int>(std::max(ncgp_sol_tot, 1), o);
  pwg_off.push_back((int)pwa.size());
  P.pwa = dev_upload(pwa, o);
  P.pwg_off = dev_upload(pwg_off, o);
  P.qp = dev_alloc<int4>(qp_tot, o); P.qw = dev_alloc<int>(qw_tot, o);
  // water-water staging chunk: a multiple of 32 waters, two blocks per SM
  const int rec_words = B.opt.precision == QB_MIXED ? WatRec<true>::words : WatRec<false>::words;
  const int chunk_max = WW_STAGE_BYTES / (16 * rec_words) / 32 * 32;
  P.ww_chunk = std::max(std::min((B.max_nwat + 31) / 32 * 32, chunk_max), 32);
  // waters per block: fewer when the batch is too small to give every SM two
  // blocks (a single system of ~1000 waters: 33 blocks of 32 instead of 5)
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.opt.device);
    B.ww_wpb = WW_WPB;
    auto blocks = [&](int wpb) {
      long long t = 0;
      for (int s = 0; s < n; s++) t += (B.sysh[s].nwat + wpb - 1) / wpb;
      return t;
    };
    while (B.ww_wpb > 32 && blocks(B.ww_wpb) < 2LL * sms) B.ww_wpb /= 2;
    long long nw = 0;
    for (int s = 0; s < n; s++) nw += B.sysh[s].nwat;
    int thr = 2048;
    cudaDeviceGetAttribute(&thr, cudaDevAttrMaxThreadsPerMultiProcessor, B.opt.device);
    B.water_atom_threads = 3 * nw <= (long long)sms * thr;
    B.water_pass_zeroes = B.max_nwat > 0;
    for (int s = 0; s < n; s++)
      if (B.sysh[s].natom != B.sysh[s].nsol + 3 * B.sysh[s].nwat) B.water_pass_zeroes = false;
  }
  // the split counts are sized for the smallest chunk a tuning may choose
  B.ww_chunk_max = P.ww_chunk;
  B.ww_chunk_floor = std::max(32, std::min(P.ww_chunk, 256));
  const int nch_alloc = (std::max(B.max_nwat, 1) + B.ww_chunk_floor - 1) / B.ww_chunk_floor;
  P.ww_nch = (std::max(B.max_nwat, 1) + P.ww_chunk - 1) / P.ww_chunk;
  // source tiles per LRF block: fewer (more blocks) when the batch is too
  // small to fill the SMs twice over
  {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.opt.device);
    int tpb = LRF_TILES_PER_BLOCK;
    B.set_lrf_tpb(tpb);
    while (tpb > 1 && (long long)B.max_lrf_blocks * n < 2LL * sms) B.set_lrf_tpb(tpb /= 2);
  }
  // water-water force blocks, system by system
  {
    long long cap = 1;
    for (int s = 0; s < n; s++) cap += (B.sysh[s].nwat + 31) / 32;
    B.ww_tiles_cap = cap;
    P.ww_tiles = dev_alloc<int2>((size_t)cap, o);
    set_ww_tiles(B, B.ww_wpb);
  }
  P.ww_cap = ww_cap;
  P.ww = dev_alloc<uint16_t>((size_t)std::max(woff, 1) * ww_cap, o);
  P.ww_n = dev_alloc<int>(std::max(woff, 1), o);
  P.ww_mid = dev_alloc<int>(std::max(woff, 1), o);
  P.ww_sp = dev_alloc<int>((size_t)std::max(woff, 1) * nch_alloc, o);
  // FP64 records on every step of the FP64 engine and on the mixed engine's
  // energy steps, whose FP64 water-water kernel stages the mixed chunk size
  // (up to 2368 waters x 80 bytes)
  P.wrec = dev_alloc<float4>((size_t)std::max(woff, 1) * WatRec<false>::words, o);
  P.wrec32 = B.opt.precision == QB_MIXED ? dev_alloc<float4>((size_t)std::max(woff, 1) * WatRec<true>::words, o)
                                         : nullptr;
  // the limits (not allocations) cover every chunk size any batch may use
  const int smem64 = std::max(WW_STAGE_BYTES, P.ww_chunk * WatRec<false>::words * 16);
  CUDA_TRY(cudaFuncSetAttribute(k_nb_ww<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, WW_STAGE_BYTES));
  CUDA_TRY(cudaFuncSetAttribute(k_nb_ww<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem64));
  CUDA_TRY(cudaFuncSetAttribute(k_nb_ww<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, WW_STAGE_BYTES));
  CUDA_TRY(cudaFuncSetAttribute(k_nb_ww<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem64));
  CUDA_TRY(cudaFuncSetAttribute(k_nb_ww<false, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem64));
  CUDA_TRY(cudaFuncSetAttribute(k_nb_ww_x2<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, WW_STAGE_BYTES));
  CUDA_TRY(cudaFuncSetAttribute(k_nb_ww_x2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, WW_STAGE_BYTES));
  P.kin_nblk = std::max(1, (B.max_natom + KIN_BLOCK - 1) / KIN_BLOCK);
  P.kin = dev_alloc<double>((size_t)n * 4, o);
  P.E = dev_alloc<double>((size_t)n * QB_NE, o);
  P.EQ = dev_alloc<double>((size_t)n * MAXS * QB_NEQ, o);
  P.offd_r = dev_alloc<double>((size_t)n * MAXS, o);
  P.hist = nullptr;
  P.hist_cap = 0;
  {
    const HistRef none{nullptr, 0};
    P.hr = dev_alloc<HistRef>(1, o);
    CUDA_TRY(cudaMemcpy(P.hr, &none, sizeof none, cudaMemcpyHostToDevice));
  }
  B.watpol_smem = (size_t)B.max_nwat * (sizeof(double) + sizeof(int));   // member angles and indices
  P.wtheta = dev_alloc<double>(std::max(woff, 1), o);
  P.wshell = dev_alloc<int8_t>(std::max(woff, 1), o);
  P.wrank = dev_alloc<int>(std::max(woff, 1), o);
  P.wshn = dev_alloc<int>((size_t)n * MAX_SHELLS, o);
  if (B.any_wpol) {
    if (B.watpol_smem > 200 * 1024) fail(QB_ERR_UNSUPPORTED, "too many waters for the polarisation kernel");
    CUDA_TRY(cudaFuncSetAttribute(k_watpol_rank, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
  }
}

}  // namespace

void ensure_history(Batch &B, int nsteps) {
  // records needed: one per output/energy interval hit, plus slack
  long long need = 2;
  for (auto &S : B.sysh) {
    long long a = S.iout > 0 ? nsteps / S.iout + 2 : 2;
    long long b = S.iene > 0 ? nsteps / S.iene + 2 : 2;
    need = std::max(need, std::max(a, b));
  }
  std::vector<SysState> st(B.nsys);
  CUDA_TRY(cudaStreamSynchronize(B.stream));   // no step in flight reads the old buffer
  CUDA_TRY(cudaMemcpy(st.data(), B.P.st, sizeof(SysState) * B.nsys, cudaMemcpyDeviceToHost));
  int used = 0;
  for (auto &x : st) used = std::max(used, std::max(x.hist_n[0], x.hist_n[1]));
  long long cap = used + need;
  if (cap <= B.P.hist_cap) return;
  cap = std::max(cap, 2LL * B.P.hist_cap);   // at least twofold
  size_t rec = HIST_REC;
  double *nh = nullptr;
  CUDA_TRY(cudaMalloc(&nh, sizeof(double) * rec * cap * 2 * B.nsys));
  CUDA_TRY(cudaMemset(nh, 0, sizeof(double) * rec * cap * 2 * B.nsys));
  if (B.P.hist) {
    for (int kind = 0; kind < 2; kind++)
      for (int s = 0; s < B.nsys; s++)
        CUDA_TRY(cudaMemcpy(nh + (((size_t)kind * B.nsys + s) * cap) * rec,
                            B.P.hist + (((size_t)kind * B.nsys + s) * B.P.hist_cap) * rec,
                            sizeof(double) * rec * B.P.hist_cap, cudaMemcpyDeviceToDevice));
    for (auto &p : B.owned)
      if (p == B.P.hist) { cudaFree(p); p = nh; }
  } else {
    B.owned.push_back(nh);
  }
  B.P.hist = nh;
  B.P.hist_cap = (int)cap;
  // the kernels read the buffer through P.hr: the captured graphs stay valid
  const HistRef ref{nh, (int)cap};
  CUDA_TRY(cudaMemcpy(B.P.hr, &ref, sizeof ref, cudaMemcpyHostToDevice));
}

// Energy-record counts of every system back to zero.
void clear_history(Batch &B) {
  std::vector<SysState> st(B.nsys);
  CUDA_TRY(cudaStreamSynchronize(B.stream));
  CUDA_TRY(cudaMemcpy(st.data(), B.P.st, sizeof(SysState) * B.nsys, cudaMemcpyDeviceToHost));
  for (auto &x : st) x.hist_n[0] = x.hist_n[1] = 0;
  CUDA_TRY(cudaMemcpy(B.P.st, st.data(), sizeof(SysState) * B.nsys, cudaMemcpyHostToDevice));
}

template <class F>
int guarded_batch(F &&f) {
  try {
    f();
    return QB_OK;
  } catch (const Error &e) {
    set_error(e.what());
    return e.code;
  } catch (const std::exception &e) {
    set_error(e.what());
    return QB_ERR_ARG;
  }
}

}  // namespace qb

namespace qb {
namespace {
// FMA throughput probe: 8 independent FMA chains per thread.
template <class T>
__global__ void k_fma_peak(T *out, int iters, T a, T b) {
  T x[8];
  for (int k = 0; k < 8; k++) x[k] = (T)(threadIdx.x + k);
  for (int it = 0; it < iters; it++)
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = x[k] * a + b;
  T s = 0;
  for (int k = 0; k < 8; k++) s += x[k];
  if (s == (T)-1.2345) out[0] = s;
}
}  // namespace
}  // namespace qb

struct qb_batch {
  qb::Batch b;
};

using qb::Batch;
using qb::guarded_batch;

extern "C" {

int qb_device_count(int *out) {
  if (!out) return QB_ERR_ARG;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) n = 0;
  *out = n;
  return QB_OK;
}

int qb_batch_create(qb_handle *const *systems, int n, const qb_options *opt, qb_batch **out) {
  if (!systems || n <= 0 || !out) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  *out = nullptr;
  qb_batch *b = new qb_batch();
  int rc = guarded_batch([&] {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) qb::fail(QB_ERR_CUDA, "no CUDA device available");
    if (opt) b->b.opt = *opt;
    CUDA_TRY(cudaSetDevice(b->b.opt.device));
    if (b->b.opt.precision != QB_FP64 && b->b.opt.precision != QB_MIXED) qb::fail(QB_ERR_ARG, "unknown precision");
    CUDA_TRY(cudaStreamCreateWithFlags(&b->b.stream, cudaStreamNonBlocking));
    b->b.use_graphs = std::getenv("QB_NO_GRAPHS") == nullptr;
    if (std::getenv("QB_ONE_STREAM") == nullptr) b->b.make_side_streams();
    qb::build(b->b, systems, n);
    // md_run's initial temperature (md.f90:3960-3963)
    qb::k_kinetic<<<dim3(b->b.P.kin_nblk, n), qb::KIN_BLOCK, 0, b->b.stream>>>(b->b.P);
    qb::k_finish<<<n, 32, 0, b->b.stream>>>(b->b.P, 0);
    b->b.check_launch("initial temperature");
    CUDA_TRY(cudaStreamSynchronize(b->b.stream));
  });
  if (rc != QB_OK) { delete b; return rc; }
  *out = b;
  return QB_OK;
}

namespace qb {
namespace {

void reset_counters(Batch &B) {
  k_reset_counters<<<Batch::cdiv(B.nsys, 128), 128, 0, B.stream>>>(B.P);
  B.check_launch("reset_counters");
}

// Work totals of the current lists and SHAKE statistics of the last run.
void refresh_workload(Batch &B, int nsteps) {
  std::vector<SysState> st(B.nsys);
  CUDA_TRY(cudaMemcpy(st.data(), B.P.st, sizeof(SysState) * B.nsys, cudaMemcpyDeviceToHost));
  std::vector<int> wwn(std::max(B.P.nwat_tot, 1));
  CUDA_TRY(cudaMemcpy(wwn.data(), B.P.ww_n, sizeof(int) * wwn.size(), cudaMemcpyDeviceToHost));
  double ww = 0;
  for (int k = 0; k < B.P.nwat_tot; k++) ww += wwn[k];
  double pw = 0, pp = 0, qp = 0, qw = 0, sh = 0, cg = B.P.ncgp_tot, its = 0, itmax = 0;
  for (int s = 0; s < B.nsys; s++) {
    pp += st[s].pp_n; pw += st[s].pw_n; qp += (double)st[s].qp_n * B.sysh[s].S;
    qw += (double)st[s].qw_n * B.sysh[s].nq * B.sysh[s].S;
    sh += B.views[s].shake_constraints;
    its += (double)st[s].shake_its;
    itmax = std::max(itmax, (double)st[s].shake_its_max);
  }
  double w[QB_WORKLOAD_N] = {ww / 2, pw, pp, qp, qw, (double)B.P.natoms_tot, sh, cg,
                             B.P.nshake_tot > 0 && nsteps > 0 ? its / ((double)B.P.nshake_tot * nsteps) : 0.0,
                             itmax};
  std::memcpy(B.workload, w, sizeof w);
}

}  // namespace
}  // namespace qb

int qb_batch_run(qb_batch *bb, int nsteps) {
  if (!bb || nsteps < 0) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    CUDA_TRY(cudaSetDevice(B.opt.device));
    qb::ensure_history(B, nsteps);
    qb::reset_counters(B);
    B.steps(nsteps);
    if (B.profiling) B.collect();
    B.sync_status();
    qb::refresh_workload(B, nsteps);
  });
}

int qb_batch_run_timed(qb_batch *bb, int nsteps, double *device_ms, long long *kernel_launches) {
  if (!bb || nsteps < 0) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    CUDA_TRY(cudaSetDevice(B.opt.device));
    qb::ensure_history(B, nsteps);
    qb::reset_counters(B);
    qb::EventPair ev;
    long long l0 = B.launches;
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    CUDA_TRY(cudaEventRecord(ev.e[0], B.stream));
    B.steps(nsteps);
    CUDA_TRY(cudaEventRecord(ev.e[1], B.stream));
    CUDA_TRY(cudaEventSynchronize(ev.e[1]));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]));
    if (device_ms) *device_ms = ms;
    if (kernel_launches) *kernel_launches = B.launches - l0;
    if (B.profiling) B.collect();
    B.sync_status();
    qb::refresh_workload(B, nsteps);
  });
}

namespace qb {
namespace {

void get_tuning(const Batch &B, qb_tuning *t) {
  t->lrf_tiles_per_block = B.P.lrf_tpb;
  t->ww_chunk = B.P.ww_chunk;
  t->side_streams = B.streams_on ? 1 : 0;
  t->ww_waters_per_block = B.ww_wpb;
  t->water_pass_per_atom = B.water_atom_threads ? 1 : 0;
  t->ww_chunk_min = B.ww_chunk_floor;
  t->ww_chunk_max = B.ww_chunk_max;
}

void set_tuning(Batch &B, const qb_tuning &t) {
  if (t.lrf_tiles_per_block < 1 || t.lrf_tiles_per_block > 1024) fail(QB_ERR_ARG, "lrf_tiles_per_block out of range");
  if (t.ww_chunk % 32 || t.ww_chunk < B.ww_chunk_floor || t.ww_chunk > B.ww_chunk_max)
    fail(QB_ERR_ARG, "ww_chunk must be a multiple of 32 within the batch's range");
  if (t.ww_waters_per_block % 32 || t.ww_waters_per_block < 32 || t.ww_waters_per_block > WW_WPB)
    fail(QB_ERR_ARG, "ww_waters_per_block must be a multiple of 32 from 32 to 256");
  if (t.water_pass_per_atom != 0 && t.water_pass_per_atom != 1) fail(QB_ERR_ARG, "water_pass_per_atom must be 0 or 1");
  CUDA_TRY(cudaStreamSynchronize(B.stream));
  B.drop_graphs();
  B.set_lrf_tpb(t.lrf_tiles_per_block);
  B.P.ww_chunk = t.ww_chunk;
  B.P.ww_nch = (std::max(B.max_nwat, 1) + t.ww_chunk - 1) / t.ww_chunk;
  B.streams_on = t.side_streams != 0;
  if (t.ww_waters_per_block != B.ww_wpb) set_ww_tiles(B, t.ww_waters_per_block);
  B.water_atom_threads = t.water_pass_per_atom != 0;
  B.lists_stale = true;   // the water-water split counts depend on the chunk
}

// device ms per step of `steps` steps after one list cycle of warm-up
double time_steps(Batch &B, int steps) {
  for (int k = 0; k < B.NB; k++) B.step();
  EventPair ev;
  CUDA_TRY(cudaEventRecord(ev.e[0], B.stream));
  B.steps(steps);
  CUDA_TRY(cudaEventRecord(ev.e[1], B.stream));
  CUDA_TRY(cudaEventSynchronize(ev.e[1]));
  float ms = 0;
  CUDA_TRY(cudaEventElapsedTime(&ms, ev.e[0], ev.e[1]));
  B.sync_status();
  return ms / steps;
}

}  // namespace
}  // namespace qb

int qb_batch_get_tuning(qb_batch *bb, qb_tuning *out) {
  if (!bb || !out) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  std::memset(out, 0, sizeof *out);
  qb::get_tuning(bb->b, out);
  return QB_OK;
}

int qb_batch_set_tuning(qb_batch *bb, const qb_tuning *t) {
  if (!bb || !t) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    CUDA_TRY(cudaSetDevice(bb->b.opt.device));
    qb::set_tuning(bb->b, *t);
  });
}

int qb_batch_autotune(qb_batch *bb, int steps_per_trial, qb_tuning *out) {
  if (!bb || steps_per_trial <= 0) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    CUDA_TRY(cudaSetDevice(B.opt.device));
    const int steps = (steps_per_trial + B.NB - 1) / B.NB * B.NB;
    qb::ensure_history(B, steps + B.NB);
    qb_tuning best{};
    qb::get_tuning(B, &best);
    int trials = 0;
    auto run = [&](const qb_tuning &t) {
      qb::set_tuning(B, t);
      trials++;
      double ms = qb::time_steps(B, steps);
      qb::clear_history(B);
      return ms;
    };
    const double before = run(best);
    double best_ms = before;
    auto consider = [&](qb_tuning t) {
      double ms = run(t);
      if (ms < best_ms) { best_ms = ms; best = t; }
    };
    if (B.any_lrf)
      for (int tpb : {1, 2, 8, 16, 4}) {
        qb_tuning t = best;
        t.lrf_tiles_per_block = tpb;
        if (tpb != best.lrf_tiles_per_block) consider(t);
      }
    if (B.max_nwat > 0)
      for (int div : {2, 4}) {
        qb_tuning t = best;
        const int c = (B.ww_chunk_max / div + 31) / 32 * 32;
        if (c < B.ww_chunk_floor || c == best.ww_chunk) continue;
        t.ww_chunk = c;
        consider(t);
      }
    if (B.max_nwat > 0)
      for (int wpb : {64, 32, 128, 192, qb::WW_WPB}) {
        qb_tuning t = best;
        t.ww_waters_per_block = wpb;
        if (wpb != best.ww_waters_per_block) consider(t);
      }
    if (B.max_nwat > 0) {
      qb_tuning t = best;
      t.water_pass_per_atom = !best.water_pass_per_atom;
      consider(t);
    }
    if (B.side[0]) {
      qb_tuning t = best;
      t.side_streams = !best.side_streams;
      consider(t);
    }
    qb::set_tuning(B, best);
    best.trials = trials;
    best.ms_per_step = best_ms;
    best.ms_per_step_before = before;
    if (out) *out = best;
  });
}

int qb_batch_fep(qb_batch *bb, const int *sys, int nfiles, const qb_fep_params *p, qb_fep_result *out) {
  if (!bb || !sys || !p || nfiles < 1) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    CUDA_TRY(cudaSetDevice(B.opt.device));
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    std::vector<qb::SysState> st(B.nsys);
    CUDA_TRY(cudaMemcpy(st.data(), B.P.st, sizeof(qb::SysState) * B.nsys, cudaMemcpyDeviceToHost));
    // energy-file records (kind 1) of each system, read in place in the ring
    const long long rec_len = qb::HIST_REC;
    qb::FepSource src;
    src.base = B.P.hist;
    src.rec_stride = (int)rec_len;
    for (int f = 0; f < nfiles; f++) {
      const int s = sys[f];
      if (s < 0 || s >= B.nsys) qb::fail(QB_ERR_ARG, "system index out of range");
      const int ns = B.sysh[s].S;
      if (f == 0) src.nstates = ns;
      else if (ns != src.nstates) qb::fail(QB_ERR_ARG, "systems with different numbers of states");
      if (!B.P.hist) qb::fail(QB_ERR_STATE, "no energy records: run the batch first");
      src.foff.push_back((((long long)B.nsys + s) * B.P.hist_cap) * rec_len + 1 + QB_NE);
      src.npts.push_back(std::min(st[s].hist_n[1], B.P.hist_cap));
      // EVB: the first off-diagonal function's r_kl of each record
      if (p->nnoffd > 0 && B.views[s].noffd < p->nnoffd)
        qb::fail(QB_ERR_ARG, "system " + std::to_string(s) + " has fewer off-diagonal functions than requested");
      src.rfoff.push_back((((long long)B.nsys + s) * B.P.hist_cap) * rec_len + 1 + QB_NE + qb::MAXS * QB_NEQ);
    }
    src.rbase = B.P.hist;
    src.r_stride = (int)rec_len;
    qb::fep_run(src, *p, B.opt.device, B.stream, out);
  });
}

int qb_batch_evaluate(qb_batch *bb, int energies) {
  if (!bb || (energies != 0 && energies != 1)) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    CUDA_TRY(cudaSetDevice(B.opt.device));
    B.build_lists(1);
    B.pot_energy(B.opt.precision == QB_MIXED ? energies : 1);
    qb::k_finish<<<B.nsys, 32, 0, B.stream>>>(B.P, 2);
    B.check_launch("energy sums");
    B.sync_status();
  });
}

int qb_batch_final_energy(qb_batch *bb) { return qb_batch_evaluate(bb, 1); }

static int sys_check(qb_batch *bb, int sys) {
  if (!bb || sys < 0 || sys >= bb->b.nsys) { qb::set_error("invalid batch or system index"); return QB_ERR_ARG; }
  return QB_OK;
}

int qb_batch_energies(qb_batch *bb, int sys, double *E_out, double *EQ_out) {
  if (int rc = sys_check(bb, sys)) return rc;
  return guarded_batch([&] {
    Batch &B = bb->b;
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    if (E_out) CUDA_TRY(cudaMemcpy(E_out, B.P.E + (size_t)sys * QB_NE, sizeof(double) * QB_NE, cudaMemcpyDeviceToHost));
    if (EQ_out && B.sysh[sys].S > 0)
      CUDA_TRY(cudaMemcpy(EQ_out, B.P.EQ + (size_t)sys * qb::MAXS * QB_NEQ, sizeof(double) * QB_NEQ * B.sysh[sys].S,
                          cudaMemcpyDeviceToHost));
  });
}

int qb_batch_temperature(qb_batch *bb, int sys, double *out) {
  if (int rc = sys_check(bb, sys)) return rc;
  return guarded_batch([&] {
    qb::SysState st;
    CUDA_TRY(cudaStreamSynchronize(bb->b.stream));
    CUDA_TRY(cudaMemcpy(&st, bb->b.P.st + sys, sizeof st, cudaMemcpyDeviceToHost));
    out[0] = st.Temp; out[1] = st.Tfree; out[2] = st.Tfree_sol; out[3] = st.Tfree_solv; out[4] = st.Tscale_solv;
  });
}

static int get_vec(qb_batch *bb, int sys, double4 *src, double *out) {
  if (int rc = sys_check(bb, sys)) return rc;
  if (!out) { qb::set_error("null buffer"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    const qb::SysDev &S = B.sysh[sys];
    std::vector<double4> tmp(S.natom);
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    CUDA_TRY(cudaMemcpy(tmp.data(), src + S.aoff, sizeof(double4) * S.natom, cudaMemcpyDeviceToHost));
    for (int i = 0; i < S.natom; i++) { out[3 * i] = tmp[i].x; out[3 * i + 1] = tmp[i].y; out[3 * i + 2] = tmp[i].z; }
  });
}

static int set_vec(qb_batch *bb, int sys, double4 *dst, const double *in) {
  if (int rc = sys_check(bb, sys)) return rc;
  if (!in) { qb::set_error("null buffer"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    const qb::SysDev &S = B.sysh[sys];
    std::vector<double4> tmp(S.natom);
    for (int i = 0; i < S.natom; i++) tmp[i] = make_double4(in[3 * i], in[3 * i + 1], in[3 * i + 2], 0);
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    CUDA_TRY(cudaMemcpy(dst + S.aoff, tmp.data(), sizeof(double4) * S.natom, cudaMemcpyHostToDevice));
  });
}

int qb_batch_gradient(qb_batch *b, int sys, double *d) { return get_vec(b, sys, b ? b->b.P.d : nullptr, d); }
int qb_batch_get_coords(qb_batch *b, int sys, double *x) { return get_vec(b, sys, b ? b->b.P.x : nullptr, x); }
int qb_batch_set_coords(qb_batch *b, int sys, const double *x) {
  int rc = set_vec(b, sys, b ? b->b.P.x : nullptr, x);
  if (rc == QB_OK) b->b.lists_stale = true;   // new coordinates: lists and LRF rebuilt before the next step
  return rc;
}
int qb_batch_get_velocities(qb_batch *b, int sys, double *v) { return get_vec(b, sys, b ? b->b.P.v : nullptr, v); }
int qb_batch_set_velocities(qb_batch *b, int sys, const double *v) { return set_vec(b, sys, b ? b->b.P.v : nullptr, v); }

// x, y, z of every atom between the engine's double4 arrays and a packed
// device copy of the caller's layout: the host copies move the packed 24
// bytes per atom (from the caller's buffer directly; page-locked buffers go
// at full link speed) and the device does the repacking.
__global__ void k_xyz_to_atoms(double4 *dst, const double *src, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = make_double4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.0);
}
__global__ void k_atoms_to_xyz(double *dst, const double4 *src, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    const double4 a = src[i];
    dst[3 * i] = a.x; dst[3 * i + 1] = a.y; dst[3 * i + 2] = a.z;
  }
}

static double *xyz_scratch(Batch &B) {
  if (!B.xyz) B.xyz = qb::dev_alloc<double>(3 * (size_t)std::max(B.P.natoms_tot, 1), B.owned);
  return B.xyz;
}

static int get_all(qb_batch *bb, double4 *src, double *out) {
  if (!bb || !out) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    const int n = B.P.natoms_tot;
    double *d = xyz_scratch(B);
    B.launches++;
    k_atoms_to_xyz<<<Batch::cdiv(n, 256), 256, 0, B.stream>>>(d, src, n);
    B.check_launch("atoms_to_xyz");
    CUDA_TRY(cudaMemcpyAsync(out, d, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, B.stream));
    CUDA_TRY(cudaStreamSynchronize(B.stream));
  });
}

static int set_all(qb_batch *bb, double4 *dst, const double *in) {
  if (!bb || !in) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    const int n = B.P.natoms_tot;
    double *d = xyz_scratch(B);
    CUDA_TRY(cudaMemcpyAsync(d, in, 3 * (size_t)n * sizeof(double), cudaMemcpyHostToDevice, B.stream));
    B.launches++;
    k_xyz_to_atoms<<<Batch::cdiv(n, 256), 256, 0, B.stream>>>(dst, d, n);
    B.check_launch("xyz_to_atoms");
    CUDA_TRY(cudaStreamSynchronize(B.stream));
  });
}

int qb_batch_get_coords_all(qb_batch *b, double *x) { return get_all(b, b ? b->b.P.x : nullptr, x); }
int qb_batch_set_coords_all(qb_batch *b, const double *x) {
  int rc = set_all(b, b ? b->b.P.x : nullptr, x);
  if (rc == QB_OK) b->b.lists_stale = true;
  return rc;
}
int qb_batch_get_velocities_all(qb_batch *b, double *v) { return get_all(b, b ? b->b.P.v : nullptr, v); }
int qb_batch_set_velocities_all(qb_batch *b, const double *v) { return set_all(b, b ? b->b.P.v : nullptr, v); }

int qb_batch_history_all(qb_batch *bb, int kind, int max_records, int *counts, double *records, size_t *bytes) {
  if (!bb || kind < 0 || kind > 1 || max_records < 0 || !counts) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    const int n = B.nsys, cap = B.P.hist_cap;
    static_assert(QB_HIST_REC == qb::HIST_REC, "record layout");
    const size_t rec = qb::HIST_REC;
    const size_t st_bytes = sizeof(qb::SysState) * n;
    // the first m records of every system: one strided copy of n rows
    const int m = records ? std::min(max_records, cap) : 0;
    const size_t row = (size_t)m * rec * sizeof(double);
    char *h = static_cast<char *>(B.staging(st_bytes + row * n));
    CUDA_TRY(cudaMemcpyAsync(h, B.P.st, st_bytes, cudaMemcpyDeviceToHost, B.stream));
    if (m > 0)
      CUDA_TRY(cudaMemcpy2DAsync(h + st_bytes, row, B.P.hist + (size_t)kind * n * cap * rec, (size_t)cap * rec * sizeof(double),
                                 row, n, cudaMemcpyDeviceToHost, B.stream));
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    if (bytes) *bytes = st_bytes + row * n;
    const qb::SysState *st = reinterpret_cast<const qb::SysState *>(h);
    const double *hr = reinterpret_cast<const double *>(h + st_bytes);
    for (int s2 = 0; s2 < n; s2++) {
      const int have = std::min(st[s2].hist_n[kind], cap);
      const int c = records ? std::min(have, m) : have;
      counts[s2] = c;
      if (records && c > 0)
        std::memcpy(records + (size_t)s2 * max_records * rec, hr + (size_t)s2 * m * rec, sizeof(double) * rec * c);
    }
  });
}

int qb_batch_step_count(qb_batch *bb, long long *out) {
  if (!bb || !out) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  *out = bb->b.istep;
  return QB_OK;
}

int qb_batch_box(qb_batch *bb, int sys, double *box6, long long *tries, long long *accepted) {
  if (int rc = sys_check(bb, sys)) return rc;
  if (!box6) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    qb::SysState st;
    CUDA_TRY(cudaStreamSynchronize(bb->b.stream));
    CUDA_TRY(cudaMemcpy(&st, bb->b.P.st + sys, sizeof st, cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3; k++) { box6[k] = st.boxl[k]; box6[3 + k] = st.boxc[k]; }
    const bool have = bb->b.mc.size() > (size_t)sys;
    if (tries) *tries = have ? bb->b.mc[sys].tries : 0;
    if (accepted) *accepted = have ? bb->b.mc[sys].accepted : 0;
  });
}

int qb_batch_get_theta_corr(qb_batch *bb, int sys, float *out, int n) {
  if (int rc = sys_check(bb, sys)) return rc;
  return guarded_batch([&] {
    qb::SysState st;
    CUDA_TRY(cudaStreamSynchronize(bb->b.stream));
    CUDA_TRY(cudaMemcpy(&st, bb->b.P.st + sys, sizeof st, cudaMemcpyDeviceToHost));
    for (int k = 0; k < n && k < qb::MAX_SHELLS; k++) out[k] = st.theta_corr[k];
  });
}

int qb_batch_history(qb_batch *bb, int sys, int kind, int *count, int *steps, double *E, double *EQ) {
  if (int rc = sys_check(bb, sys)) return rc;
  if (kind < 0 || kind > 1 || !count) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    qb::SysState st;
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    CUDA_TRY(cudaMemcpy(&st, B.P.st + sys, sizeof st, cudaMemcpyDeviceToHost));
    int c = std::min(st.hist_n[kind], B.P.hist_cap);
    *count = c;
    if (c == 0 || (!steps && !E && !EQ)) return;
    size_t rec = qb::HIST_REC;
    std::vector<double> h(rec * c);
    CUDA_TRY(cudaMemcpy(h.data(), B.P.hist + (((size_t)kind * B.nsys + sys) * B.P.hist_cap) * rec,
                        sizeof(double) * rec * c, cudaMemcpyDeviceToHost));
    int S = B.sysh[sys].S;
    for (int r = 0; r < c; r++) {
      const double *p = h.data() + rec * r;
      if (steps) steps[r] = (int)p[0];
      if (E) std::memcpy(E + (size_t)r * QB_NE, p + 1, sizeof(double) * QB_NE);
      if (EQ && S > 0) std::memcpy(EQ + (size_t)r * S * QB_NEQ, p + 1 + QB_NE, sizeof(double) * S * QB_NEQ);
    }
  });
}

int qb_batch_offdiag(qb_batch *bb, int sys, int kind, int *count, double *out) {
  if (int rc = sys_check(bb, sys)) return rc;
  if (kind < 0 || kind > 2 || !count) { qb::set_error("invalid argument"); return QB_ERR_ARG; }
  return guarded_batch([&] {
    Batch &B = bb->b;
    qb::SysState st;
    CUDA_TRY(cudaStreamSynchronize(B.stream));
    CUDA_TRY(cudaMemcpy(&st, B.P.st + sys, sizeof st, cudaMemcpyDeviceToHost));
    const qb_sysview &V = B.views[sys];
    // kind 2: the values of the latest force evaluation, as one record
    int c = kind == 2 ? 1 : std::min(st.hist_n[kind], B.P.hist_cap);
    *count = c;
    if (c == 0 || !out || V.noffd == 0) return;
    size_t rec = qb::HIST_REC, roff = 1 + QB_NE + qb::MAXS * QB_NEQ;
    std::vector<double> h(rec * c);
    if (kind == 2)
      CUDA_TRY(cudaMemcpy(h.data() + roff, B.P.offd_r + (size_t)sys * qb::MAXS, sizeof(double) * qb::MAXS,
                          cudaMemcpyDeviceToHost));
    else
      CUDA_TRY(cudaMemcpy(h.data(), B.P.hist + (((size_t)kind * B.nsys + sys) * B.P.hist_cap) * rec,
                          sizeof(double) * rec * c, cudaMemcpyDeviceToHost));
    for (int r = 0; r < c; r++)
      for (int io = 0; io < V.noffd; io++) {
        double rkl = h[rec * r + roff + io];
        out[((size_t)r * V.noffd + io) * 2] = V.offd_A[io] * std::exp(-V.offd_mu[io] * rkl);
        out[((size_t)r * V.noffd + io) * 2 + 1] = rkl;
      }
  });
}

int qb_batch_clear_history(qb_batch *bb) {
  if (!bb) return QB_ERR_ARG;
  return guarded_batch([&] { qb::clear_history(bb->b); });
}

int qb_batch_status(qb_batch *bb, int sys, int *status) {
  if (int rc = sys_check(bb, sys)) return rc;
  return guarded_batch([&] {
    qb::SysState st;
    CUDA_TRY(cudaStreamSynchronize(bb->b.stream));
    CUDA_TRY(cudaMemcpy(&st, bb->b.P.st + sys, sizeof st, cudaMemcpyDeviceToHost));
    *status = st.status;
  });
}

int qb_batch_set_profiling(qb_batch *bb, int on) {
  if (!bb) return QB_ERR_ARG;
  bb->b.profiling = on != 0;
  if (on) { bb->b.stats.clear(); bb->b.order.clear(); }
  return QB_OK;
}

int qb_batch_profile(qb_batch *bb, char *names, size_t names_len, double *ms, long long *launches, int n,
                     int *n_kernels) {
  if (!bb) return QB_ERR_ARG;
  Batch &B = bb->b;
  std::string all;
  int k = 0;
  for (auto &name : B.order) {
    if (k < n) {
      if (ms) ms[k] = B.stats[name].ms;
      if (launches) launches[k] = B.stats[name].launches;
      all += name + "\n";
    }
    k++;
  }
  if (names && names_len) std::snprintf(names, names_len, "%s", all.c_str());
  if (n_kernels) *n_kernels = k;
  return QB_OK;
}

int qb_batch_workload(qb_batch *bb, double *out, int n) {
  if (!bb || !out) return QB_ERR_ARG;
  for (int k = 0; k < n && k < QB_WORKLOAD_N; k++) out[k] = bb->b.workload[k];
  return QB_OK;
}

void qb_batch_destroy(qb_batch *bb) { delete bb; }


int qb_peak_flops(int device, int precision, double *tflops) {
  if (!tflops) return QB_ERR_ARG;
  return guarded_batch([&] {
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    int blocks = prop.multiProcessorCount * 8, threads = 256, iters = 1 << 14;
    void *buf = nullptr;
    CUDA_TRY(cudaMalloc(&buf, 64));
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
      CUDA_TRY(cudaEventRecord(e0));
      if (precision == QB_FP64)
        qb::k_fma_peak<double><<<blocks, threads>>>((double *)buf, iters, 0.999999, 1e-7);
      else
        qb::k_fma_peak<float><<<blocks, threads>>>((float *)buf, iters, 0.999999f, 1e-7f);
      CUDA_TRY(cudaEventRecord(e1));
      CUDA_TRY(cudaEventSynchronize(e1));
      float ms;
      CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0) best = std::min(best, ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    double flop = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flop / (best * 1e-3) / 1e12;
  });
}

}  // extern "C"
