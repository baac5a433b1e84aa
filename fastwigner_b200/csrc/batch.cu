// Persistent batched Moyal propagation over instances with uneven grids.
//
// One cooperative launch advances every instance by `steps` steps.  The
// launch walks a fixed phase list -- opening V/2 column pass, then per step a
// row pass (K) and a fused column pass (V/2, observables, V/2 of the next step),
// then a normalisation phase -- and separates phases with a software grid
// barrier.  Inside a phase the CTAs pull (instance, tile) work items from an
// atomic queue and run the size-specialised tile code of wigner_tiles.cuh for
// that instance's P (column items) or X (row items), so 128^2 and 1024^2
// instances share the machine in one launch.  Every spin in the barrier has an
// iteration limit: on expiry the kernel records FW_BATCH_TIMEOUT in the status
// word and all CTAs return.
#include <cuda_runtime.h>
#include <math.h>
#include <string>
#include <vector>
#include <algorithm>
#include "wigner_tiles.cuh"
#include "fw_internal.h"

namespace fw {

struct BatchInst {
  float* W;
  int P, X;
  const void* tabV;
  const void* tabK;
  const void* twP;
  const void* twX;
  double dxdp;
  double* part;       // 2 slots x ncol x 2
  int ncol;           // column tiles per instance (partial records)
  int nrow;           // row work items per instance
};

struct BatchArgs {
  const BatchInst* inst;
  int ninst;
  const int2* col_items;  // (instance, tile)
  int ncol_items;
  const int2* row_items;
  int nrow_items;
  int steps;
  double* obs;            // steps x ninst x 2
  int* counters;          // one work counter per phase (zeroed before launch)
  unsigned int* barrier;  // [arrive count, generation]
  int* status;
  long long spin_limit;
};

constexpr int BT = 256;   // threads per CTA of the persistent kernel
constexpr int BM = 2;     // observables per step: sum W, sum W^2

// launch shapes per size (variant 0: 32 values per thread at 1024; variant 1: 16)
template <int N, int V> struct BCol;
template <int N, int V> struct BRow;
template <int V> struct BCol<128, V> { static constexpr int T = 16, CP = 16; };
template <int V> struct BCol<256, V> { static constexpr int T = 32, CP = 8; };
template <int V> struct BCol<512, V> { static constexpr int T = (V == 0 ? 32 : 64), CP = BT / T; };
template <int V> struct BCol<1024, V> { static constexpr int T = (V == 0 ? 32 : 64), CP = BT / T; };
template <int V> struct BRow<128, V> { static constexpr int T = 16, G = 16; };
template <int V> struct BRow<256, V> { static constexpr int T = 32, G = 8; };
template <int V> struct BRow<512, V> { static constexpr int T = (V == 0 ? 32 : 64), G = BT / T; };
template <int V> struct BRow<1024, V> { static constexpr int T = (V == 0 ? 32 : 64), G = BT / T; };

// The persistent kernel records no p-observables (Mp = 0), so its column
// tiles never touch the per-bin sum buffer that follows the exchange buffer:
// the exchange buffer alone is allocated (keeps three CTAs per SM possible).
template <int N, int V> constexpr size_t bcol_smem() {
  return col_ex_reals<float, N, BCol<N, V>::T, BCol<N, V>::CP>() * sizeof(float);
}
template <int N, int V> constexpr size_t brow_smem() {
  return (size_t)BRow<N, V>::G * 2 * (N + N / 32) * sizeof(float);
}
template <int V> constexpr size_t batch_smem() {
  size_t m = 0;
  m = std::max(m, bcol_smem<128, V>()); m = std::max(m, bcol_smem<256, V>());
  m = std::max(m, bcol_smem<512, V>()); m = std::max(m, bcol_smem<1024, V>());
  m = std::max(m, brow_smem<128, V>()); m = std::max(m, brow_smem<256, V>());
  m = std::max(m, brow_smem<512, V>()); m = std::max(m, brow_smem<1024, V>());
  return m;
}

// Bounded sense-reversal grid barrier; returns false when the launch must stop.
__device__ __forceinline__ bool grid_sync(const BatchArgs& a, int* sflag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vb = a.barrier;
    const unsigned int gen = vb[1];
    __threadfence();
    const unsigned int arrived = atomicAdd(&a.barrier[0], 1u) + 1u;
    if (arrived == gridDim.x) {
      a.barrier[0] = 0u;
      __threadfence();
      atomicAdd(&a.barrier[1], 1u);
    } else {
      long long it = 0;
      while (vb[1] == gen) {
        if (*(volatile int*)a.status != 0) break;
        if (++it > a.spin_limit) {
          atomicCAS(a.status, 0, FW_BATCH_TIMEOUT);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    *sflag = *(volatile int*)a.status;
  }
  __syncthreads();
  return *sflag == 0;
}

template <int V>
__device__ __forceinline__ void do_col(const BatchArgs& a, const BatchInst& in, int tile, int k, bool open,
                                       unsigned char* smem, double* red, double (*ored)[2 + 2 * MAXO]) {
  PassArgs p{};
  p.W = in.W;
  p.P = in.P;
  p.X = in.X;
  p.batch = 1;
  p.scale_const = 1.0;
  p.dxdp = in.dxdp;
  p.out_scale = 1.0;
  p.M = BM;
  p.tab1 = in.tabV;
  p.tw = in.twP;
  if (!open) {
    p.part_out = in.part + (size_t)(k & 1) * in.ncol * BM;
    if (k + 1 < a.steps) {
      p.tab2 = in.tabV;
      p.fuse_mid = 1;
    }
  }
  switch (in.P) {
#define COLN(N_)                                                                                            \
  case N_: {                                                                                                \
    constexpr int T = BCol<N_, V>::T, CP = BCol<N_, V>::CP;                                                 \
    col_tile<float, N_, T, CP>(p, 0, tile, in.ncol, smem, red, ored);                                        \
  } break;
    COLN(128) COLN(256) COLN(512) COLN(1024)
#undef COLN
  }
}

template <int V>
__device__ __forceinline__ void do_row(const BatchArgs& a, const BatchInst& in, int blk, int k, unsigned char* smem,
                                       double* red, int inst_index) {
  PassArgs p{};
  p.W = in.W;
  p.P = in.P;
  p.X = in.X;
  p.batch = 1;
  p.scale_const = 1.0;
  p.dxdp = in.dxdp;
  p.out_scale = 1.0;
  p.M = BM;
  p.tab1 = in.tabK;
  p.tw = in.twX;
  if (k > 0) {
    p.prev_part = in.part + (size_t)((k - 1) & 1) * in.ncol * BM;
    p.prev_nparts = in.ncol;
    if (a.obs) p.obs_hist = a.obs + ((size_t)(k - 1) * a.ninst + inst_index) * BM;
  }
  switch (in.X) {
#define ROWN(N_)                                                              \
  case N_: {                                                                  \
    constexpr int T = BRow<N_, V>::T, G = BRow<N_, V>::G;                     \
    row_tile<float, N_, T, G>(p, 0, blk, smem, red);                          \
  } break;
    ROWN(128) ROWN(256) ROWN(512) ROWN(1024)
#undef ROWN
  }
}

template <int V>
__global__ void __launch_bounds__(BT, 1) batch_moyal_kernel(BatchArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double red[34];
  __shared__ double ored[BT / 32][2 + 2 * MAXO];
  __shared__ int item;
  __shared__ int sflag;
  int phase = 0;
  auto run_phase = [&](int n_items, auto&& body) {
    for (;;) {
      __syncthreads();
      if (threadIdx.x == 0) item = atomicAdd(&a.counters[phase], 1);
      __syncthreads();
      const int it = item;
      if (it >= n_items) break;
      body(it);
    }
    ++phase;
  };
  // opening V/2 of step 0
  run_phase(a.ncol_items, [&](int it) {
    const int2 w = a.col_items[it];
    do_col<V>(a, a.inst[w.x], w.y, 0, true, smem, red, ored);
  });
  if (!grid_sync(a, &sflag)) return;
  for (int k = 0; k < a.steps; ++k) {
    run_phase(a.nrow_items, [&](int it) {
      const int2 w = a.row_items[it];
      do_row<V>(a, a.inst[w.x], w.y, k, smem, red, w.x);
    });
    if (!grid_sync(a, &sflag)) return;
    run_phase(a.ncol_items, [&](int it) {
      const int2 w = a.col_items[it];
      do_col<V>(a, a.inst[w.x], w.y, k, false, smem, red, ored);
    });
    if (!grid_sync(a, &sflag)) return;
  }
  // final normalisation: one item per (instance, row block), scale from the last partials
  run_phase(a.nrow_items, [&](int it) {
    const int2 w = a.row_items[it];
    const BatchInst& in = a.inst[w.x];
    PassArgs p{};
    p.prev_part = in.part + (size_t)((a.steps - 1) & 1) * in.ncol * BM;
    p.prev_nparts = in.ncol;
    p.M = BM;
    p.dxdp = in.dxdp;
    if (a.obs) p.obs_hist = a.obs + ((size_t)(a.steps - 1) * a.ninst + w.x) * BM;
    const double sc = prev_scale(p, 0, red, w.y == 0);
    const int rows_per = in.P / in.nrow;
    float* W = in.W + (size_t)w.y * rows_per * in.X;
    const size_t n = (size_t)rows_per * in.X;
    for (size_t i = threadIdx.x; i < n; i += blockDim.x) W[i] = (float)(__ldcg(W + i) * sc);
  });
}

}  // namespace fw

using namespace fw;

struct fw_batch {
  int ninst = 0;
  int variant = 0;
  std::vector<BatchInst> host_inst;
  BatchInst* dev_inst = nullptr;
  int2* dev_col = nullptr;
  int2* dev_row = nullptr;
  int ncol_items = 0, nrow_items = 0;
  void* tw[4] = {nullptr, nullptr, nullptr, nullptr};  // twiddles for 128, 256, 512, 1024
  double* part = nullptr;
  int* counters = nullptr;
  int counters_cap = 0;
  unsigned int* barrier = nullptr;
  int* status = nullptr;
  long long spin_limit = 1LL << 25;  // polls per barrier wait (~2-4 s) before the launch gives up
  int grid = 0;
  bool dirty = true;
  // CUDA graph of the last propagate(steps, obs)
  cudaGraphExec_t gexec = nullptr;
  int g_steps = -1;
  double* g_obs = nullptr;
  cudaStream_t g_stream = nullptr;
};

namespace {
int size_index(int n) { return n == 128 ? 0 : n == 256 ? 1 : n == 512 ? 2 : n == 1024 ? 3 : -1; }

template <int N, int V> int col_cp() { return BCol<N, V>::CP; }
template <int N, int V> int row_g() { return BRow<N, V>::G; }
int col_cp_of(int N, int v) {
  switch (N) {
    case 128: return v ? col_cp<128, 1>() : col_cp<128, 0>();
    case 256: return v ? col_cp<256, 1>() : col_cp<256, 0>();
    case 512: return v ? col_cp<512, 1>() : col_cp<512, 0>();
    default: return v ? col_cp<1024, 1>() : col_cp<1024, 0>();
  }
}
int row_g_of(int N, int v) {
  switch (N) {
    case 128: return v ? row_g<128, 1>() : row_g<128, 0>();
    case 256: return v ? row_g<256, 1>() : row_g<256, 0>();
    case 512: return v ? row_g<512, 1>() : row_g<512, 0>();
    default: return v ? row_g<1024, 1>() : row_g<1024, 0>();
  }
}

int upload_tw32(int n, void** dev) {
  std::vector<float> t(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    const double ang = -2.0 * M_PI * (double)k / (double)n;
    t[2 * k] = (float)cos(ang);
    t[2 * k + 1] = (float)sin(ang);
  }
  cudaError_t e = cudaMalloc(dev, t.size() * sizeof(float));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(batch twiddles)");
  e = cudaMemcpy(*dev, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(batch twiddles)");
  return FW_OK;
}

template <int V> const void* kernel_ptr() { return (const void*)batch_moyal_kernel<V>; }
template <int V> size_t kernel_smem() { return batch_smem<V>(); }

int release_graph(fw_batch* b) {
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  b->gexec = nullptr;
  b->g_steps = -1;
  return FW_OK;
}

// (re)build work lists, per-instance partial slots and the launch grid
int prepare(fw_batch* b) {
  if (!b->dirty) return FW_OK;
  std::vector<int2> col, row;
  size_t part_doubles = 0;
  for (int i = 0; i < b->ninst; ++i) {
    BatchInst& in = b->host_inst[i];
    if (in.W == nullptr || in.tabV == nullptr || in.tabK == nullptr)
      return fail(FW_ESTATE, "fw_batch: instance " + std::to_string(i) + " has no state or tables");
    in.ncol = in.X / (2 * col_cp_of(in.P, b->variant));
    in.nrow = (in.P / 2) / row_g_of(in.X, b->variant);
    in.twP = b->tw[size_index(in.P)];
    in.twX = b->tw[size_index(in.X)];
    part_doubles += (size_t)2 * in.ncol * BM;
  }
  // larger instances first so the queue tail is made of small items
  std::vector<int> order(b->ninst);
  for (int i = 0; i < b->ninst; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    return (long long)b->host_inst[x].P * b->host_inst[x].X > (long long)b->host_inst[y].P * b->host_inst[y].X;
  });
  for (int i : order) {
    for (int t = 0; t < b->host_inst[i].ncol; ++t) col.push_back(make_int2(i, t));
    for (int t = 0; t < b->host_inst[i].nrow; ++t) row.push_back(make_int2(i, t));
  }
  cudaFree(b->part);
  cudaFree(b->dev_col);
  cudaFree(b->dev_row);
  cudaFree(b->dev_inst);
  b->part = nullptr; b->dev_col = b->dev_row = nullptr; b->dev_inst = nullptr;
  cudaError_t e = cudaMalloc(&b->part, part_doubles * sizeof(double));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(batch partials)");
  size_t off = 0;
  for (int i = 0; i < b->ninst; ++i) {
    b->host_inst[i].part = b->part + off;
    off += (size_t)2 * b->host_inst[i].ncol * BM;
  }
  if ((e = cudaMalloc(&b->dev_col, col.size() * sizeof(int2))) != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  if ((e = cudaMalloc(&b->dev_row, row.size() * sizeof(int2))) != cudaSuccess) return cuda_fail(e, "cudaMalloc");
  if ((e = cudaMalloc(&b->dev_inst, b->host_inst.size() * sizeof(BatchInst))) != cudaSuccess)
    return cuda_fail(e, "cudaMalloc");
  cudaMemcpy(b->dev_col, col.data(), col.size() * sizeof(int2), cudaMemcpyHostToDevice);
  cudaMemcpy(b->dev_row, row.data(), row.size() * sizeof(int2), cudaMemcpyHostToDevice);
  cudaMemcpy(b->dev_inst, b->host_inst.data(), b->host_inst.size() * sizeof(BatchInst), cudaMemcpyHostToDevice);
  b->ncol_items = (int)col.size();
  b->nrow_items = (int)row.size();
  // persistent grid: every CTA resident (cooperative launch)
  const void* kp = b->variant ? kernel_ptr<1>() : kernel_ptr<0>();
  const size_t smem = b->variant ? kernel_smem<1>() : kernel_smem<0>();
  e = cudaFuncSetAttribute(kp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(batch kernel)");
  int per_sm = 0, dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kp, BT, smem);
  if (e != cudaSuccess || per_sm < 1) return fail(FW_ECUDA, "fw_batch: persistent kernel does not fit on an SM");
  b->grid = per_sm * sms;
  b->dirty = false;
  release_graph(b);
  return FW_OK;
}

int launch(fw_batch* b, int steps, double* obs, cudaStream_t st) {
  const int nphase = 2 * steps + 2;
  if (nphase > b->counters_cap) {
    cudaFree(b->counters);
    b->counters = nullptr;
    cudaError_t e = cudaMalloc(&b->counters, sizeof(int) * (size_t)nphase);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(batch counters)");
    b->counters_cap = nphase;
    release_graph(b);
  }
  cudaError_t e = cudaMemsetAsync(b->counters, 0, sizeof(int) * (size_t)nphase, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->barrier, 0, 2 * sizeof(unsigned int), st);
  if (e != cudaSuccess) return cuda_fail(e, "batch counter reset");
  BatchArgs a{};
  a.inst = b->dev_inst;
  a.ninst = b->ninst;
  a.col_items = b->dev_col;
  a.ncol_items = b->ncol_items;
  a.row_items = b->dev_row;
  a.nrow_items = b->nrow_items;
  a.steps = steps;
  a.obs = obs;
  a.counters = b->counters;
  a.barrier = b->barrier;
  a.status = b->status;
  a.spin_limit = b->spin_limit;
  void* args[] = {&a};
  const void* kp = b->variant ? kernel_ptr<1>() : kernel_ptr<0>();
  const size_t smem = b->variant ? kernel_smem<1>() : kernel_smem<0>();
  e = cudaLaunchCooperativeKernel(kp, dim3(b->grid), dim3(BT), args, smem, st);
  if (e != cudaSuccess) return cuda_fail(e, "batch cooperative launch");
  count_launch(1);
  return FW_OK;
}
}  // namespace

extern "C" int fw_batch_num_variants(void) { return 2; }

extern "C" int fw_batch_create(int ninst, const int* P, const int* X, int variant, fw_batch** out) {
  if (out == nullptr || P == nullptr || X == nullptr || ninst < 1) return fail(FW_EINVAL, "fw_batch_create: bad arguments");
  *out = nullptr;
  if (variant < 0 || variant > 1) return fail(FW_EINVAL, "fw_batch_create: variant must be 0 or 1");
  for (int i = 0; i < ninst; ++i)
    if (size_index(P[i]) < 0 || size_index(X[i]) < 0)
      return fail(FW_EINVAL, "fw_batch_create: batched grids must be 128, 256, 512 or 1024 per axis (instance " +
                                 std::to_string(i) + ")");
  fw_batch* b = new fw_batch();
  b->ninst = ninst;
  b->variant = variant;
  b->host_inst.resize(ninst);
  for (int i = 0; i < ninst; ++i) {
    b->host_inst[i] = BatchInst{};
    b->host_inst[i].P = P[i];
    b->host_inst[i].X = X[i];
  }
  int rc = FW_OK;
  const int sizes[4] = {128, 256, 512, 1024};
  for (int s = 0; s < 4 && rc == FW_OK; ++s) rc = upload_tw32(sizes[s], &b->tw[s]);
  if (rc == FW_OK) {
    cudaError_t e = cudaMalloc(&b->barrier, 2 * sizeof(unsigned int));
    if (e == cudaSuccess) e = cudaMalloc(&b->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->status, 0, sizeof(int));
    if (e != cudaSuccess) rc = cuda_fail(e, "cudaMalloc(batch control)");
  }
  if (rc != FW_OK) {
    fw_batch_destroy(b);
    return rc;
  }
  *out = b;
  return FW_OK;
}

extern "C" int fw_batch_set_variant(fw_batch* b, int variant) {
  if (b == nullptr || variant < 0 || variant > 1) return fail(FW_EINVAL, "fw_batch_set_variant: bad arguments");
  if (b->variant != variant) {
    b->variant = variant;
    b->dirty = true;
  }
  return FW_OK;
}

extern "C" int fw_batch_set_instance(fw_batch* b, int i, void* W, const void* tabV, const void* tabK, double dxdp) {
  if (b == nullptr || i < 0 || i >= b->ninst) return fail(FW_EINVAL, "fw_batch_set_instance: bad instance");
  BatchInst& in = b->host_inst[i];
  in.W = static_cast<float*>(W);
  in.tabV = tabV;
  in.tabK = tabK;
  in.dxdp = dxdp;
  b->dirty = true;
  return FW_OK;
}

extern "C" int fw_batch_propagate(fw_batch* b, int steps, double* obs, int use_graph, void* stream) {
  if (b == nullptr) return fail(FW_EINVAL, "fw_batch_propagate: NULL batch");
  if (steps <= 0) return steps == 0 ? FW_OK : fail(FW_EINVAL, "fw_batch_propagate: steps < 0");
  int rc = prepare(b);
  if (rc != FW_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!use_graph) return launch(b, steps, obs, st);
  if (b->gexec == nullptr || b->g_steps != steps || b->g_obs != obs) {
    release_graph(b);
    if (2 * steps + 2 > b->counters_cap) {  // size the counters outside the capture
      cudaFree(b->counters);
      b->counters = nullptr;
      cudaError_t e = cudaMalloc(&b->counters, sizeof(int) * (size_t)(2 * steps + 2));
      if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(batch counters)");
      b->counters_cap = 2 * steps + 2;
    }
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreate(capture)");
    cudaGraph_t g;
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) { cudaStreamDestroy(cs); return cuda_fail(e, "cudaStreamBeginCapture"); }
    rc = launch(b, steps, obs, cs);
    e = cudaStreamEndCapture(cs, &g);
    cudaStreamDestroy(cs);
    if (rc != FW_OK) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    e = cudaGraphInstantiate(&b->gexec, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->gexec = nullptr; return cuda_fail(e, "cudaGraphInstantiate"); }
    b->g_steps = steps;
    b->g_obs = obs;
  }
  cudaError_t e = cudaGraphLaunch(b->gexec, st);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGraphLaunch");
  return FW_OK;
}

extern "C" int fw_batch_status(fw_batch* b, int* status_out) {
  if (b == nullptr || status_out == nullptr) return fail(FW_EINVAL, "fw_batch_status: NULL argument");
  cudaError_t e = cudaMemcpy(status_out, b->status, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "fw_batch_status");
  return FW_OK;
}

extern "C" int fw_batch_set_spin_limit(fw_batch* b, long long polls) {
  if (b == nullptr || polls < 0) return fail(FW_EINVAL, "fw_batch_set_spin_limit: bad arguments");
  if (b->spin_limit != polls) {
    b->spin_limit = polls;
    release_graph(b);  // a captured launch holds the old limit in its arguments
  }
  return FW_OK;
}

extern "C" int fw_batch_set_status(fw_batch* b, int status) {
  if (b == nullptr) return fail(FW_EINVAL, "fw_batch_set_status: NULL batch");
  cudaError_t e = cudaMemcpy(b->status, &status, sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "fw_batch_set_status");
  return FW_OK;
}

extern "C" int fw_batch_destroy(fw_batch* b) {
  if (b == nullptr) return FW_OK;
  release_graph(b);
  for (void* t : b->tw) cudaFree(t);
  cudaFree(b->part);
  cudaFree(b->dev_col);
  cudaFree(b->dev_row);
  cudaFree(b->dev_inst);
  cudaFree(b->counters);
  cudaFree(b->barrier);
  cudaFree(b->status);
  delete b;
  return FW_OK;
}
