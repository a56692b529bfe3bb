// ss3d_batch.cu -- batched form: many realizations of many grid shapes in one
// CUDA-graph launch.
//
// A batch is a list of jobs (spectrum, seed, first realization, count, device
// output).  Its work is captured once into a CUDA graph and ss3d_batch_run is
// one graph launch.  Two schedules, chosen by the batch autotuner:
//
//   chains      one chain per job -- row states, synthesis + first inverse
//               pass, middle pass, C2R x pass -- on parallel graph branches, so
//               the passes of small grids run beside those of large ones and a
//               job's next pass starts as soon as its own previous pass ends.
//               Each kernel is the per-call kernel with its own length-specific
//               tile (tile variants tuned per pass kind for the batch).
//   persistent  row states of all jobs, then three pass kernels, each a grid
//               sized to the resident CTAs of the GPU that walks one work list
//               holding the tiles of every job.  One CTA shape for every
//               length: 512 threads with 16 or 8 elements per thread.
//
// Every tile body is the device function of the per-call path
// (ss3d_bodies.cuh) with the same Park-Miller row states, so a batched
// realization equals the same realization computed alone, bit for bit.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/specsim3d_gpu.h"
#include "ss3d_bodies.cuh"

namespace ss3d {

extern int g_variant[3][2][16];

constexpr int BNT = 512;
constexpr int BL_MIN = 4, BL_MAX = 10;   // column passes of the persistent schedule: lengths 16 .. 1024
constexpr int BR_MIN = 3, BR_MAX = 9;    // its row pass: npx/2 = 8 .. 512
constexpr int NETV = 2;                  // persistent tile variants: 16 or 8 elements per thread
__host__ __device__ constexpr int et_of(int v) { return v == 0 ? 16 : 8; }

// uniform persistent tile of length 2^L: BNT threads, ET elements per thread
template <int L, int ETV> struct BCfg {
  static constexpr int N = 1 << L;
  static constexpr int ET = N < et_of(ETV) ? N : et_of(ETV);
  static constexpr int TPC = N / ET;
  static constexpr int TX = BNT / TPC;
  static_assert(TX * TPC == BNT, "uniform batch tile");
};
__host__ __device__ constexpr int tx_of(int L, int etv) {
  return BNT / ((1 << L) < et_of(etv) ? 1 : (1 << L) / et_of(etv));
}
// dynamic shared memory of the bodies (complex float elements of 8 bytes)
constexpr size_t smem_col(int L, int etv) { return (size_t)((1 << L) * tx_of(L, etv) + (1 << L)) * 8; }
constexpr size_t smem_row(int L, int etv) {
  return (size_t)(((1 << L) + 1) * (tx_of(L, etv) + 1) + 3 * (1 << L)) * 8;
}

struct BJob {
  Geo g;
  const float* amp;
  const uint32_t* rs;
  const uint32_t* apow;
  float2* work;
  long long wstride;
  float* out;
  int nreal;
  int pad_;
  AxisArgs A, B;       // first and middle pass geometry (tpg of the chosen tile)
  int LA, LB, LC;      // log2 transform lengths, -1 when the pass is absent
  int start[3];        // first work item of this job in each pass
  int count[3];        // work items of this job in each pass
  int pad2_;
};

template <int PASS, int ETV>
__device__ __forceinline__ void run_item(const BJob& J, int local, const Tw& tw, unsigned char* sm) {
  const Geo g = J.g;
  if constexpr (PASS == 0) {
    const AxisArgs A = J.A;
    switch (J.LA) {
#define SS3D_BA(L)                                                                                          \
  case L:                                                                                                   \
    if (g.d == 2)                                                                                           \
      colgen_body<float, L, BCfg<L, ETV>::TX, BCfg<L, ETV>::TPC, 1>(A, g, J.amp, J.rs, J.apow, J.work, tw, \
                                                                    local, sm);                            \
    else                                                                                                    \
      colgen_body<float, L, BCfg<L, ETV>::TX, BCfg<L, ETV>::TPC, 0>(A, g, J.amp, J.rs, J.apow, J.work, tw, \
                                                                    local, sm);                            \
    break;
      SS3D_BA(4) SS3D_BA(5) SS3D_BA(6) SS3D_BA(7) SS3D_BA(8) SS3D_BA(9) SS3D_BA(10)
#undef SS3D_BA
      default: break;
    }
  } else if constexpr (PASS == 1) {
    const AxisArgs B = J.B;
    switch (J.LB) {
#define SS3D_BB(L)                                                                                    \
  case L:                                                                                             \
    col_body<float, L, BCfg<L, ETV>::TX, BCfg<L, ETV>::TPC, +1>(B, g, J.work, J.work, tw, local, sm); \
    break;
      SS3D_BB(4) SS3D_BB(5) SS3D_BB(6) SS3D_BB(7) SS3D_BB(8) SS3D_BB(9) SS3D_BB(10)
#undef SS3D_BB
      default: break;
    }
  } else {
    const long long ostride = (long long)g.nx * g.ny * g.nz;
    switch (J.LC) {
#define SS3D_BC(L)                                                                                         \
  case L:                                                                                                  \
    rows_body<float, float, L, BCfg<L, ETV>::TX, BCfg<L, ETV>::TPC>(g, J.work, J.wstride, J.out, ostride, \
                                                                    J.nreal, 0, nullptr, tw, local, sm);  \
    break;
      SS3D_BC(3) SS3D_BC(4) SS3D_BC(5) SS3D_BC(6) SS3D_BC(7) SS3D_BC(8) SS3D_BC(9)
#undef SS3D_BC
      default: break;
    }
  }
}

// Persistent pass kernel over the work items of all jobs.  chunk = 0: CTAs
// stride over the items by the grid size; chunk > 0: CTA b takes items
// [b*chunk, (b+1)*chunk) in order.  Items only increase within a CTA, so the
// job index only advances: every thread finds it the same way (a binary
// search for the first item, then forward steps), and warp 0 copies the job
// descriptor into shared memory when it changes.
template <int PASS, int ETV>
__global__ void __launch_bounds__(BNT, ETV == 1 ? 2 : 1)
    k_batch_pass(const BJob* __restrict__ jobs, int njobs, int total, int chunk, Tw tw) {
  extern __shared__ __align__(16) unsigned char smb[];
  __shared__ __align__(16) BJob J;
  constexpr int NWORD = sizeof(BJob) / 4;
  static_assert(sizeof(BJob) % 4 == 0, "job descriptor copied in words");
  int item, end, step;
  if (chunk > 0) {
    item = blockIdx.x * chunk;
    end = min(total, item + chunk);
    step = 1;
  } else {
    item = blockIdx.x;
    end = total;
    step = gridDim.x;
  }
  if (item >= end) return;
  int lo = 0, hi = njobs - 1;   // last job whose first item is <= item
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].start[PASS] <= item) lo = mid;
    else hi = mid - 1;
  }
  int j = lo, jcur = -1;
  for (; item < end; item += step) {
    while (j + 1 < njobs && jobs[j + 1].start[PASS] <= item) ++j;
    if (j != jcur) {
      if (threadIdx.x < 32) {
        const uint32_t* src = reinterpret_cast<const uint32_t*>(jobs + j);
        uint32_t* dst = reinterpret_cast<uint32_t*>(&J);
        for (int w = threadIdx.x; w < NWORD; w += 32) dst[w] = __ldg(src + w);
      }
      __syncthreads();
      jcur = j;
    }
    run_item<PASS, ETV>(J, item - J.start[PASS], tw, smb);
    __syncthreads();   // shared memory and J are reused by the next item
  }
}

using BatchKernel = void (*)(const BJob*, int, int, int, Tw);
const BatchKernel kBatchKernels[3][NETV] = {{k_batch_pass<0, 0>, k_batch_pass<0, 1>},
                                            {k_batch_pass<1, 0>, k_batch_pass<1, 1>},
                                            {k_batch_pass<2, 0>, k_batch_pass<2, 1>}};

const void* module_anchor_batch() { return reinterpret_cast<const void*>(kBatchKernels[0][0]); }

}  // namespace ss3d

using namespace ss3d;

struct ss3d_batch {
  int dev = 0;
  int nsm = 148;
  std::vector<BJob> jobs;
  BJob* djobs = nullptr;
  std::vector<void*> bufs;
  int sched = 0;             // 0 chains, 1 persistent
  // chains: tile variant per pass kind (0 middle, 1 synthesis, 2 rows) and length
  int var[3][16] = {};
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr;
  // chains: realizations of a job split into this many consecutive sub-chains,
  // each starting its synthesis when the previous one's synthesis has ended
  int split = 1;
  std::vector<cudaEvent_t> stag;   // synthesis-done events of the sub-chains
  // persistent: per pass
  int etv[3] = {0, 0, 0};    // tile variant
  int mode[3] = {0, 0, 0};   // 0 strided items, 1 contiguous items, 2 one CTA per item
  int cps[3] = {0, 0, 0};    // CTAs per SM (0: occupancy limit)
  int chunk[3] = {0, 0, 0};
  int total[3] = {0, 0, 0};
  int grid[3] = {0, 0, 0};
  size_t smem[3] = {0, 0, 0};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool pipes = false;        // the graph holds kernels with bounded bulk-copy waits
  Tw tw{};
  const uint32_t* ptab = nullptr;
  std::vector<uint32_t> s0;
  std::vector<long long> r_first;
  long long cells = 0;
  int kernels = 0;           // kernel nodes of the captured graph
};

namespace {
int ilog2b(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

bool persistent_ok(const BJob& J) {
  return J.LA >= BL_MIN && J.LA <= BL_MAX && (J.LB < 0 || (J.LB >= BL_MIN && J.LB <= BL_MAX)) && J.LC >= BR_MIN &&
         J.LC <= BR_MAX;
}
bool all_persistent_ok(const ss3d_batch* b) {
  for (const BJob& J : b->jobs)
    if (!persistent_ok(J)) return false;
  return true;
}

// Persistent schedule: work lists, shared memory and grids for the chosen tile
// variants; uploads the job table.
cudaError_t plan(ss3d_batch* b) {
  int start[3] = {0, 0, 0};
  size_t sm[3] = {0, 0, 0};
  for (BJob& J : b->jobs) {
    const int txA = tx_of(J.LA, b->etv[0]);
    J.A.tpg = (J.A.lines + txA - 1) / txA;
    J.count[0] = J.A.tpg * J.A.ngroups * J.nreal;
    sm[0] = std::max(sm[0], smem_col(J.LA, b->etv[0]));
    J.count[1] = 0;
    if (J.LB >= 0) {
      const int txB = tx_of(J.LB, b->etv[1]);
      J.B.tpg = (J.B.lines + txB - 1) / txB;
      J.count[1] = J.B.tpg * J.B.ngroups * J.nreal;
      sm[1] = std::max(sm[1], smem_col(J.LB, b->etv[1]));
    }
    const int txC = tx_of(J.LC, b->etv[2]);
    J.count[2] = ((J.g.ny * J.g.nz + txC - 1) / txC) * J.nreal;
    sm[2] = std::max(sm[2], smem_row(J.LC, b->etv[2]));
    for (int p = 0; p < 3; p++) {
      J.start[p] = start[p];
      start[p] += J.count[p];
    }
  }
  cudaError_t e = cudaMemcpy(b->djobs, b->jobs.data(), sizeof(BJob) * b->jobs.size(), cudaMemcpyHostToDevice);
  for (int p = 0; p < 3 && e == cudaSuccess; p++) {
    b->total[p] = start[p];
    b->smem[p] = sm[p];
    b->grid[p] = 0;
    if (!start[p]) continue;
    BatchKernel k = kBatchKernels[p][b->etv[p]];
    e = func_smem(reinterpret_cast<const void*>(k), sm[p]);
    int occ = 0;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k, BNT, sm[p]);
    if (e == cudaSuccess && occ < 1) e = cudaErrorInvalidConfiguration;
    const int cps = b->cps[p] > 0 ? std::min(b->cps[p], occ) : occ;
    if (b->mode[p] == 2) {
      b->grid[p] = start[p];
      b->chunk[p] = 0;
    } else {
      b->grid[p] = std::max(1, std::min(start[p], b->nsm * cps));
      b->chunk[p] = b->mode[p] == 1 ? (start[p] + b->grid[p] - 1) / b->grid[p] : 0;
    }
  }
  return e;
}

// Persistent schedule on stream st; with ev, events before each pass and after
// the last (ev[0] .. ev[3]).
cudaError_t enqueue_persistent(ss3d_batch* b, cudaStream_t st, cudaEvent_t* ev) {
  cudaError_t e = cudaSuccess;
  for (size_t j = 0; j < b->jobs.size() && e == cudaSuccess; j++) {
    const BJob& J = b->jobs[j];
    e = launch_rowstates(J.g, b->s0[j], b->r_first[j], J.nreal, b->ptab, const_cast<uint32_t*>(J.rs),
                         const_cast<uint32_t*>(J.apow), st);
  }
  for (int p = 0; p < 3 && e == cudaSuccess; p++) {
    if (ev) e = cudaEventRecord(ev[p], st);
    if (e != cudaSuccess || !b->total[p]) continue;
    kBatchKernels[p][b->etv[p]]<<<b->grid[p], BNT, b->smem[p], st>>>(b->djobs, (int)b->jobs.size(), b->total[p],
                                                                     b->chunk[p], b->tw);
    ++g_launch_count;
    e = cudaGetLastError();
  }
  if (ev && e == cudaSuccess) e = cudaEventRecord(ev[3], st);
  return e;
}

// Chains schedule: sub-chain c (realizations r0..r1 of one job: row states,
// synthesis, middle and row passes) on branch stream c mod B, forked from and
// joined back into st.  With split S a job's realizations form S consecutive
// sub-chains, and sub-chain q starts only when the synthesis of sub-chain q-1
// has ended: the syntheses, bound by instruction issue, then run one after
// the other while the memory-bound middle and row passes of the earlier
// sub-chains run beside them.  The per-call launchers pick their tile from
// g_variant, set to the batch's choice for the duration of the enqueue.
cudaError_t enqueue_chains(ss3d_batch* b, cudaStream_t st) {
  int saved[3][16];
  for (int k = 0; k < 3; k++)
    for (int L = 0; L < 16; L++) {
      saved[k][L] = g_variant[k][1][L];
      g_variant[k][1][L] = b->var[k][L];
    }
  const int nb = (int)b->branch.size();
  cudaError_t e = cudaSuccess;
  size_t nstag = 0;
  for (const BJob& J : b->jobs) nstag += (size_t)std::max(0, std::min(b->split, J.nreal) - 1);
  while (b->stag.size() < nstag && e == cudaSuccess) {
    cudaEvent_t ev = nullptr;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) b->stag.push_back(ev);
  }
  if (e == cudaSuccess) e = cudaEventRecord(b->fork, st);
  for (int q = 0; q < nb && e == cudaSuccess; q++) e = cudaStreamWaitEvent(b->branch[q], b->fork, 0);
  int chain = 0;
  size_t ist = 0;
  for (size_t j = 0; j < b->jobs.size() && e == cudaSuccess; j++) {
    const BJob& J = b->jobs[j];
    const int S = std::min(b->split, J.nreal);
    const long long rows = (long long)J.g.npy * J.g.npz, M = (long long)J.g.nx * J.g.ny * J.g.nz;
    cudaEvent_t prev = nullptr;
    for (int q = 0; q < S && e == cudaSuccess; q++, chain++) {
      const int r0 = (int)((long long)J.nreal * q / S), r1 = (int)((long long)J.nreal * (q + 1) / S);
      cudaStream_t s = b->branch[chain % nb];
      cudaEvent_t done = q + 1 < S ? b->stag[ist++] : nullptr;
      if (prev) e = cudaStreamWaitEvent(s, prev, 0);
      // the column offsets a^(d i) are written once, by the first sub-chain
      if (e == cudaSuccess)
        e = launch_rowstates(J.g, b->s0[j], b->r_first[j] + r0, r1 - r0, b->ptab,
                             const_cast<uint32_t*>(J.rs) + r0 * rows, q == 0 ? const_cast<uint32_t*>(J.apow) : nullptr,
                             s);
      if (e == cudaSuccess)
        e = launch_realize<float>(J.g, J.amp, J.rs + r0 * rows, J.apow, J.work + r0 * J.wstride, J.wstride, r1 - r0,
                                  J.out + r0 * M, 0, nullptr, nullptr, b->tw, true, s, nullptr, done);
      prev = done;
    }
  }
  for (int q = 0; q < nb && e == cudaSuccess; q++) {
    e = cudaEventRecord(b->joins[q], b->branch[q]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(st, b->joins[q], 0);
  }
  for (int k = 0; k < 3; k++)
    for (int L = 0; L < 16; L++) g_variant[k][1][L] = saved[k][L];
  return e;
}

cudaError_t enqueue(ss3d_batch* b, cudaStream_t st, cudaEvent_t* ev = nullptr) {
  if (b->sched == 1) return enqueue_persistent(b, st, ev);
  cudaError_t e = ev ? cudaEventRecord(ev[0], st) : cudaSuccess;
  if (e == cudaSuccess) e = enqueue_chains(b, st);
  if (ev)
    for (int q = 1; q < 4 && e == cudaSuccess; q++) e = cudaEventRecord(ev[q], st);
  return e;
}

int capture(ss3d_batch* b) {
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaStream_t cs;
  cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  if (e != cudaSuccess) return set_error(SS3D_ECUDA, cudaGetErrorString(e));
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    const unsigned long long pipes0 = g_pipe_launches.load();
    cudaError_t e2 = enqueue(b, cs);
    b->pipes = g_pipe_launches.load() != pipes0;
    e = cudaStreamEndCapture(cs, &b->graph);
    if (e2 != cudaSuccess) e = e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  size_t nn = 0;
  if (e == cudaSuccess) {
    std::vector<cudaGraphNode_t> nodes;
    e = cudaGraphGetNodes(b->graph, nullptr, &nn);
    if (e == cudaSuccess && nn) {
      nodes.resize(nn);
      e = cudaGraphGetNodes(b->graph, nodes.data(), &nn);
    }
    int nk = 0;
    for (size_t q = 0; q < nn && e == cudaSuccess; q++) {
      cudaGraphNodeType t;
      e = cudaGraphNodeGetType(nodes[q], &t);
      if (t == cudaGraphNodeTypeKernel) ++nk;
    }
    b->kernels = nk;
  }
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) return set_error(SS3D_ECUDA, (std::string("batch graph: ") + cudaGetErrorString(e)).c_str());
  return SS3D_OK;
}

int cuda_err(cudaError_t e, const char* what) {
  return set_error(e == cudaErrorMemoryAllocation ? SS3D_ENOMEM : SS3D_ECUDA,
                   (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

// one timed run of the current schedule (after a warm-up run); pass times in
// ms[0..2] (persistent only, else -1) and the whole run in ms[3]
cudaError_t time_run(ss3d_batch* b, cudaStream_t st, float ms[4], bool warm) {
  cudaEvent_t ev[4] = {};
  cudaError_t e = cudaSuccess;
  for (int q = 0; q < 4 && e == cudaSuccess; q++) e = cudaEventCreate(&ev[q]);
  if (e == cudaSuccess && warm) e = enqueue(b, st);
  if (e == cudaSuccess) e = enqueue(b, st, ev);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev[3]);
  for (int p = 0; p < 3 && e == cudaSuccess; p++) {
    e = cudaEventElapsedTime(&ms[p], ev[p], ev[p + 1]);
    if (b->sched == 0) ms[p] = -1.f;
  }
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms[3], ev[0], ev[3]);
  for (int q = 0; q < 4; q++)
    if (ev[q]) cudaEventDestroy(ev[q]);
  return e;
}
}  // namespace

extern "C" void ss3d_batch_free(ss3d_batch* b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (cudaStream_t s : b->branch) cudaStreamDestroy(s);
  for (cudaEvent_t ev : b->joins) cudaEventDestroy(ev);
  for (cudaEvent_t ev : b->stag) cudaEventDestroy(ev);
  if (b->fork) cudaEventDestroy(b->fork);
  for (void* p : b->bufs) cudaFree(p);
  if (b->djobs) cudaFree(b->djobs);
  delete b;
}

extern "C" int ss3d_batch_create(const ss3d_batch_job* jobs, int njobs, ss3d_batch** out) {
  if (!jobs || njobs < 1 || !out) return set_error(SS3D_EINVAL, "invalid batch arguments");
  *out = nullptr;
  ss3d_batch* b = new ss3d_batch();
  if (cudaGetDevice(&b->dev) != cudaSuccess) {
    delete b;
    return set_error(SS3D_ECUDA, "no CUDA device");
  }
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->dev);
  if (int rc = batch_ctx(b->dev, &b->tw, &b->ptab)) {
    delete b;
    return rc;
  }
  for (int k = 0; k < 3; k++)
    for (int L = 0; L < 16; L++) b->var[k][L] = g_variant[k][1][L];
  cudaError_t e = cudaSuccess;
  for (int j = 0; j < njobs; j++) {
    const ss3d_batch_job& q = jobs[j];
    BJob J{};
    const float* amp32 = nullptr;
    if (!q.sp || q.nreal < 1 || q.r_first < 0 || (q.igauss != 0 && q.igauss != 1) || !q.out ||
        batch_geo(q.sp, q.igauss, &J.g, &amp32)) {
      ss3d_batch_free(b);
      return set_error(SS3D_EINVAL, "invalid batch job (NULL spectrum or output, nreal < 1, r_first < 0, "
                                    "igauss not 0/1, or spectrum of another device)");
    }
    const Geo& g = J.g;
    bool dev_out = false;
    if (int rc = check_ptr(q.out, b->dev, g.nx % 2 == 0 ? 8 : 4, "batch job output", &dev_out)) {
      ss3d_batch_free(b);
      return rc;
    }
    if (!dev_out) {
      ss3d_batch_free(b);
      return set_error(SS3D_EINVAL, "batch job output must be device memory");
    }
    J.amp = amp32;
    J.nreal = q.nreal;
    J.out = q.out;
    J.LA = J.LB = J.LC = -1;
    if (g.npz > 1) {
      J.LA = ilog2b(g.npz);
      if (g.npy > 1) J.LB = ilog2b(g.npy);
    } else if (g.npy > 1) {
      J.LA = ilog2b(g.npy);
    }
    if (g.npx > 1) J.LC = ilog2b(g.npx) - 1;
    if (ilog2b(g.npx) - 1 > MAX_LOGN_F || ilog2b(g.npy) > MAX_LOGN_F || ilog2b(g.npz) > MAX_LOGN_F) {
      ss3d_batch_free(b);
      return set_error(SS3D_ETOOLARGE, "periodic axis longer than the supported transform length");
    }
    // complex work grids [r][k < nz][j < npy][HP]: the first pass stores k < nz only
    const long long wstride = (long long)(g.npz > 1 ? g.nz : 1) * g.npy * g.HP;
    AxisArgs A{};
    if (g.npz > 1) {
      A.S = (long long)g.npy * g.HP;
      A.nout = g.nz;
      A.lines = g.npy * g.HP;
      A.ngroups = 1;
      A.gstride = 0;
      A.axis = 2;
    } else {
      A.S = g.HP;
      A.nout = g.ny;
      A.lines = g.H;
      A.ngroups = 1;
      A.gstride = (long long)g.npy * g.HP;
      A.axis = 1;
    }
    A.rstride = wstride;
    A.nreal = q.nreal;
    J.A = A;
    if (J.LB >= 0) {
      AxisArgs B{};
      B.S = g.HP;
      B.nout = g.ny;
      B.lines = g.H;
      B.ngroups = g.nz;
      B.gstride = (long long)g.npy * g.HP;
      B.rstride = wstride;
      B.nreal = q.nreal;
      B.axis = 1;
      J.B = B;
    }
    uint32_t *rs = nullptr, *ap = nullptr;
    float2* work = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&rs, sizeof(uint32_t) * (size_t)g.npy * g.npz * q.nreal);
    if (e == cudaSuccess) e = cudaMalloc(&ap, sizeof(uint32_t) * g.npx);
    if (e == cudaSuccess) e = cudaMalloc(&work, sizeof(float2) * (size_t)wstride * q.nreal);
    for (void* p : {(void*)rs, (void*)ap, (void*)work})
      if (p) b->bufs.push_back(p);
    J.rs = rs;
    J.apow = ap;
    J.work = work;
    J.wstride = wstride;
    b->jobs.push_back(J);
    const int64_t a = q.iseed < 0 ? -(int64_t)q.iseed : (int64_t)q.iseed;
    b->s0.push_back((uint32_t)(a % 2147483646LL + 1));
    b->r_first.push_back(q.r_first);
    b->cells += (long long)g.nx * g.ny * g.nz * q.nreal;
  }
  long long nchains = 0;
  for (const BJob& J : b->jobs) nchains += J.nreal;
  const int nbranch = (int)std::min<long long>(nchains, 16);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
  for (int q = 0; q < nbranch && e == cudaSuccess; q++) {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) b->branch.push_back(s);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) b->joins.push_back(ev);
  }
  if (e == cudaSuccess) e = cudaMalloc(&b->djobs, sizeof(BJob) * njobs);
  if (e == cudaSuccess && all_persistent_ok(b)) e = plan(b);
  if (e != cudaSuccess) {
    ss3d_batch_free(b);
    return cuda_err(e, "batch create");
  }
  if (int rc = capture(b)) {
    ss3d_batch_free(b);
    return rc;
  }
  *out = b;
  return SS3D_OK;
}

extern "C" int ss3d_batch_run(ss3d_batch* b) {
  if (!b || !b->exec) return set_error(SS3D_EINVAL, "batch is NULL");
  cudaStream_t st = current_stream();
  cudaError_t e = cudaGraphLaunch(b->exec, st);
  g_launch_count += (unsigned long long)b->kernels;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_err(e, "batch run");
  if (b->pipes && pipe_error_take(st))
    return set_error(SS3D_ECUDA, "batch run: a bulk-copy wait of the middle pass timed out");
  return SS3D_OK;
}

extern "C" int ss3d_batch_info(const ss3d_batch* b, int64_t* cells, int grid[3], int items[3], int* kernels) {
  if (!b) return set_error(SS3D_EINVAL, "batch is NULL");
  if (cells) *cells = b->cells;
  if (kernels) *kernels = b->kernels;
  for (int p = 0; p < 3; p++) {
    if (grid) grid[p] = b->sched == 1 ? b->grid[p] : 0;
    if (items) items[p] = b->sched == 1 ? b->total[p] : 0;
  }
  return SS3D_OK;
}

extern "C" int ss3d_batch_time(ss3d_batch* b, float ms[4]) {
  if (!b || !ms) return set_error(SS3D_EINVAL, "NULL argument");
  const cudaError_t e = time_run(b, current_stream(), ms, false);
  if (e != cudaSuccess) return cuda_err(e, "batch time");
  return SS3D_OK;
}

extern "C" int ss3d_batch_schedule(const ss3d_batch* b, int* sched, int etv[3], int mode[3], int cps[3]) {
  if (!b) return set_error(SS3D_EINVAL, "batch is NULL");
  if (sched) *sched = b->sched;
  for (int p = 0; p < 3; p++) {
    if (etv) etv[p] = b->etv[p];
    if (mode) mode[p] = b->mode[p];
    if (cps) cps[p] = b->cps[p];
  }
  return SS3D_OK;
}

extern "C" int ss3d_batch_split(const ss3d_batch* b, int* split) {
  if (!b || !split) return set_error(SS3D_EINVAL, "NULL argument");
  *split = b->split;
  return SS3D_OK;
}

extern "C" int ss3d_batch_set_split(ss3d_batch* b, int split) {
  if (!b || split < 1) return set_error(SS3D_EINVAL, "invalid batch split");
  b->split = split;
  return capture(b);
}

extern "C" int ss3d_batch_set_schedule(ss3d_batch* b, int sched, int pass, int etv, int mode, int cps) {
  if (!b || sched < 0 || sched > 1 || pass < 0 || pass > 2 || etv < 0 || etv >= NETV || mode < 0 || mode > 2 ||
      cps < 0)
    return set_error(SS3D_EINVAL, "invalid batch schedule");
  if (sched == 1 && !all_persistent_ok(b))
    return set_error(SS3D_EINVAL, "the persistent schedule needs periodic axes of 16..1024 nodes and npx >= 16");
  b->sched = sched;
  if (sched == 1) {
    b->etv[pass] = etv;
    b->mode[pass] = mode;
    b->cps[pass] = cps;
    const cudaError_t e = plan(b);
    if (e != cudaSuccess) return cuda_err(e, "batch schedule");
  }
  return capture(b);
}

// Batch autotuner.  Chains: for each pass kind in turn, every tile variant of
// the lengths the batch uses, timed over whole runs.  Persistent (when every
// job fits it): for each pass, every tile variant under every mode and count
// of CTAs per SM, timed around that pass.  Keeps the faster schedule and
// re-captures the graph.  Outputs do not depend on the choice.
extern "C" int ss3d_batch_autotune(ss3d_batch* b) {
  if (!b) return set_error(SS3D_EINVAL, "batch is NULL");
  cudaStream_t st = current_stream();
  cudaError_t e = cudaSuccess;
  float ms[4];
  // chains
  b->sched = 0;
  bool used[3][16] = {};
  for (const BJob& J : b->jobs) {
    const Geo& g = J.g;
    if (g.npz > 1) {
      used[1][ilog2b(g.npz)] = true;
      if (g.npy > 1) used[0][ilog2b(g.npy)] = true;
    } else if (g.npy > 1) {
      used[1][ilog2b(g.npy)] = true;
    }
    if (g.npx > 1) used[2][ilog2b(g.npx) - 1] = true;
  }
  float best_chain = 1e30f;
  for (int k : {1, 0, 2}) {
    int bestv = 0;
    float bestk = 1e30f;
    // column passes 4-7: two-line tiles; middle pass 8-9: tiles staged by
    // bulk tensor copies; row pass 4: rows held in warps, 5: middle and row
    // passes fused over a cluster, 6: two rows per lane on packed FP32
    for (int v = 0; v < (k == 2 ? 7 : (k == 0 ? 10 : 8)) && e == cudaSuccess; v++) {
      for (int L = 0; L < 16; L++)
        if (used[k][L]) b->var[k][L] = v;
      e = time_run(b, st, ms, true);
      if (e == cudaSuccess && ms[3] < bestk) {
        bestk = ms[3];
        bestv = v;
      }
    }
    for (int L = 0; L < 16; L++)
      if (used[k][L]) b->var[k][L] = bestv;
    best_chain = bestk;
  }
  // chains: split of each job's realizations into staggered sub-chains
  {
    int maxr = 1;
    for (const BJob& J : b->jobs) maxr = std::max(maxr, J.nreal);
    int bests = b->split;
    for (int sp : {1, 2, 4, 8}) {
      if (sp > maxr || e != cudaSuccess) break;
      b->split = sp;
      e = time_run(b, st, ms, true);
      if (e == cudaSuccess && ms[3] < best_chain) {
        best_chain = ms[3];
        bests = sp;
      }
    }
    b->split = bests;
  }
  // persistent
  float best_pers = 1e30f;
  if (e == cudaSuccess && all_persistent_ok(b)) {
    b->sched = 1;
    for (int p = 0; p < 3 && e == cudaSuccess; p++) {
      e = plan(b);
      if (e != cudaSuccess || !b->total[p]) continue;
      float best = 1e30f;
      int bv = b->etv[p], bm = b->mode[p], bc = b->cps[p];
      for (int v = 0; v < NETV && e == cudaSuccess; v++) {
        for (int m = 0; m < 3 && e == cudaSuccess; m++) {
          for (int c = 1; c <= (m == 2 ? 1 : 4) && e == cudaSuccess; c++) {
            b->etv[p] = v;
            b->mode[p] = m;
            b->cps[p] = c;
            e = plan(b);
            if (e != cudaSuccess) break;
            // counts beyond the occupancy limit are clamped by plan: stop there
            if (m < 2 && c > 1 && b->grid[p] < std::min(b->total[p], b->nsm * c)) break;
            e = time_run(b, st, ms, true);
            if (e == cudaSuccess && ms[p] < best) {
              best = ms[p];
              bv = v;
              bm = m;
              bc = c;
            }
          }
        }
      }
      b->etv[p] = bv;
      b->mode[p] = bm;
      b->cps[p] = bc;
    }
    if (e == cudaSuccess) e = plan(b);
    if (e == cudaSuccess) e = time_run(b, st, ms, true);
    if (e == cudaSuccess) best_pers = ms[3];
  }
  if (e != cudaSuccess) return cuda_err(e, "batch autotune");
  b->sched = best_pers < best_chain ? 1 : 0;
  return capture(b);
}
