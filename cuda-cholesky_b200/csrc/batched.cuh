// Batched factor / log det / inverse of many small SPD matrices of uneven sizes
// (included at the end of lapack.cu; uses its launch helpers).
//
// Every matrix advances one nb-wide block column per step, all matrices in
// lockstep, so one step is three grouped launches over the whole batch:
//   1. diagonal blocks: one CTA per matrix factors and inverts its block
//      (diag_factor_batched_kernel; log det accumulated per matrix);
//   2. panel solves A21 := A21 W^H, in place (a 64-wide tile holds all nb <= 64
//      columns of a row block, so a CTA reads its rows before it writes them);
//   3. lower-only trailing updates A22 -= A21 A21^H.
// The inverse (?potri) follows the single-matrix algorithm, grouped over the batch:
// all diagonal blocks inverted in one launch, the split trees of all matrices
// walked level by level (one grouped launch per height and phase), then L^H L of
// every matrix into workspace and back (a k = 0 grouped product with beta = 1).
// A matrix whose factor fails sets its info word, and every later problem of that
// matrix is skipped (per-problem stop word).
//
// The whole sequence (about 30 launches for n <= 512) is captured once into a CUDA
// graph; a run is one graph launch.  The block size nb is chosen by timing the
// candidate graphs on an identity batch of the same shapes (the autotuner), unless
// the caller fixes it.

struct __cucholbatched_st {
  CULAPACKhandle h;
  char type;                 // 'S' or 'D'
  int batch;
  int nb;
  int* d_info;               // per matrix
  double* d_logdet;          // per matrix
  void* d_w;                 // inverses of the current step's diagonal blocks
  void* d_work;              // TRTRI X blocks, then L^H L (sum of n_b^2 elements)
  std::vector<void*> d_lists;
  int persistent;            // FP64: the whole sequence is one persistent kernel (bpersist.cuh)
  int* d_next;               // its work-queue head
  double* d_wp;              // its per-CTA inverses of the diagonal blocks (wp_tiles per CTA)
  int wp_tiles;
  bool dry;                  // recording pass 1: build and upload lists, launch nothing
  bool reuse;                // recording pass 2 (under capture): reuse the uploaded lists
  size_t cursor;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

namespace {

template <typename T>
struct BatchedShape {
  bool upper;
  int batch;
  std::vector<int> n;
  std::vector<T*> a;
  std::vector<long long> lda;
  int flags;
};

// Upload a host vector into plan-owned device memory.
template <typename V>
V* upload(CUcholBatched p, const std::vector<V>& v, CUresult* rc) {
  if (v.empty()) return nullptr;
  if (p->reuse) return static_cast<V*>(p->d_lists[p->cursor++]);   // same order as pass 1
  void* d = nullptr;
  cudaError_t e = dev_malloc(&d, v.size() * sizeof(V));
  if (e == cudaSuccess) e = cudaMemcpy(d, v.data(), v.size() * sizeof(V), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    *rc = report(e, "upload", __func__, __FILE__, __LINE__);
    if (d) cudaFree(d);
    return nullptr;
  }
  p->d_lists.push_back(d);
  return static_cast<V*>(d);
}

// Grouped SIMT launch of a device problem list (tile_begin / tiles_n already set).
template <typename T>
CUresult launch_list(CULAPACKhandle h, std::vector<GemmProblem<T>>& ps, CUcholBatched p, cudaStream_t s) {
  if (ps.empty()) return CUDA_SUCCESS;
  int tiles = 0;
  for (auto& q : ps) {
    q.tiles_n = (q.n + kTile - 1) / kTile;
    q.tile_begin = tiles;
    tiles += ((q.m + kTile - 1) / kTile) * q.tiles_n;
  }
  CUresult rc = CUDA_SUCCESS;
  const GemmProblem<T>* dev = upload(p, ps, &rc);
  if (dev == nullptr) return rc == CUDA_SUCCESS ? CUDA_ERROR_OUT_OF_MEMORY : rc;
  if (p->dry) return CUDA_SUCCESS;
  GemmLaunch<T> L{};
  L.list = dev;
  L.nlist = (int)ps.size();
  return launch_dispatch<T>(h, L, tiles, ps[0].a_rs == 1 ? 0 : 1, ps[0].b_rs == 1 ? 0 : 1, s, nullptr);
}

}  // namespace

namespace {

constexpr int kBatchedMaxNb = 64;   // a 64-wide SIMT tile holds a whole panel: in-place solve

template <typename T>
CUresult record_persistent(CUcholBatched p, const BatchedShape<T>& sh, cudaStream_t s);

// Enqueue the whole batched sequence on stream s (used under stream capture).
template <typename T>
CUresult record_batched(CUcholBatched p, const BatchedShape<T>& sh, int nb, cudaStream_t s) {
  if constexpr (std::is_same<T, double>::value) {
    if (p->persistent) return record_persistent<T>(p, sh, s);
  }
  CULAPACKhandle h = p->h;
  using Smem = DiagSmem<T, kBatchedMaxNb>;
  const int B = sh.batch;
  T* W = static_cast<T*>(p->d_w);
  T* work = static_cast<T*>(p->d_work);
  int nmax = 0;
  for (int b = 0; b < B; ++b) nmax = std::max(nmax, sh.n[b]);
  auto rs_of = [&](int b) { return sh.upper ? sh.lda[b] : 1LL; };
  auto cs_of = [&](int b) { return sh.upper ? 1LL : sh.lda[b]; };
  auto at = [&](int b, long long i, long long j) { return sh.a[b] + i * rs_of(b) + j * cs_of(b); };
  if (!p->dry) {
    CUCHOL_CHECK(cudaMemsetAsync(p->d_info, 0, sizeof(int) * B, s));
    CUCHOL_CHECK(cudaMemsetAsync(p->d_logdet, 0, sizeof(double) * B, s));
  }
  const T minus_one = from_real<T>(RealOf<T>(-1)), one = from_real<T>(RealOf<T>(1));

  // ---- factor ----
  for (int j = 0; j < nmax; j += nb) {
    std::vector<DiagTask<T>> tasks;
    std::vector<GemmProblem<T>> trsm, syrk;
    for (int b = 0; b < B; ++b) {
      if (sh.n[b] <= j) continue;
      const int jb = std::min(nb, sh.n[b] - j), m = sh.n[b] - j - jb;
      T* w = W + (size_t)tasks.size() * nb * nb;
      DiagTask<T> t;
      t.a = at(b, j, j); t.rs = rs_of(b); t.cs = cs_of(b); t.jb = jb;
      t.w = m > 0 ? w : nullptr; t.ldw = nb; t.info_base = j; t.info = p->d_info + b;
      t.logdet = (sh.flags & 2) ? p->d_logdet + b : nullptr;
      tasks.push_back(t);
      if (m == 0) continue;
      GemmProblem<T> q = problem<T>();
      q.a = at(b, j + jb, j); q.a_rs = rs_of(b); q.a_ks = cs_of(b);
      q.b = w; q.b_rs = 1; q.b_ks = nb; q.conj_b = 1;           // zeros above W's diagonal
      q.c = at(b, j + jb, j); q.c_rs = rs_of(b); q.c_cs = cs_of(b);   // in place
      q.m = m; q.n = jb; q.k = jb; q.stop = p->d_info + b;
      trsm.push_back(q);
      GemmProblem<T> u = problem<T>();
      u.a = at(b, j + jb, j); u.a_rs = rs_of(b); u.a_ks = cs_of(b);
      u.b = u.a; u.b_rs = u.a_rs; u.b_ks = u.a_ks; u.conj_b = 1;
      u.c = at(b, j + jb, j + jb); u.c_rs = rs_of(b); u.c_cs = cs_of(b);
      u.cin = u.c; u.cin_rs = u.c_rs; u.cin_cs = u.c_cs;
      u.alpha = minus_one; u.beta = one; u.lower_only = 1; u.real_diag = 1;
      u.m = m; u.n = m; u.k = jb; u.stop = p->d_info + b;
      syrk.push_back(u);
    }
    CUresult rc = CUDA_SUCCESS;
    const DiagTask<T>* dt = upload(p, tasks, &rc);
    if (dt == nullptr) return rc == CUDA_SUCCESS ? CUDA_ERROR_OUT_OF_MEMORY : rc;
    if (!p->dry) {
      diag_factor_batched_kernel<T, kBatchedMaxNb, kDiagThreads2>
          <<<(unsigned)tasks.size(), kDiagThreads2, Smem::bytes, s>>>(dt);
      ++h->launches;
      CUCHOL_CHECK(cudaGetLastError());
    }
    CUCHOL_CHECK_CU(launch_list<T>(h, trsm, p, s));
    CUCHOL_CHECK_CU(launch_list<T>(h, syrk, p, s));
  }
  if (!(sh.flags & 4)) return CUDA_SUCCESS;

  // ---- inverse: TRTRI (leaves, then the split trees level by level) ----
  std::vector<InvTask<T>> inv;
  std::vector<std::vector<Node>> trees(B);
  std::vector<size_t> woff(B);
  size_t off = 0;
  int height = 0;
  for (int b = 0; b < B; ++b) {
    for (int o = 0; o < sh.n[b]; o += nb) {
      InvTask<T> t;
      t.b = at(b, o, o); t.rs = rs_of(b); t.cs = cs_of(b);
      t.jb = std::min(nb, sh.n[b] - o); t.unit = 0; t.stop = p->d_info + b;
      inv.push_back(t);
    }
    height = std::max(height, build_tree(0, sh.n[b], nb, trees[b]));
    woff[b] = off;
    off += (size_t)sh.n[b] * sh.n[b];
  }
  CUresult rc = CUDA_SUCCESS;
  const InvTask<T>* di = upload(p, inv, &rc);
  if (di == nullptr) return rc == CUDA_SUCCESS ? CUDA_ERROR_OUT_OF_MEMORY : rc;
  if (!p->dry) {
    diag_invert_batched_kernel<T, kBatchedMaxNb, kDiagThreads2>
        <<<(unsigned)inv.size(), kDiagThreads2, Smem::bytes, s>>>(di);
    ++h->launches;
    CUCHOL_CHECK(cudaGetLastError());
  }
  for (int hh = 1; hh <= height; ++hh) {
    std::vector<GemmProblem<T>> p1, p2;
    for (int b = 0; b < B; ++b) {
      size_t xo = woff[b];
      for (auto& nd : trees[b]) {
        if (nd.height != hh) continue;
        const int s1 = nd.s1, s2 = nd.s - nd.s1, o = nd.o;
        T* x = work + xo;
        xo += (size_t)s2 * s1;
        GemmProblem<T> a = problem<T>();   // X = T22^-1 T21
        a.a = at(b, o + s1, o + s1); a.a_rs = rs_of(b); a.a_ks = cs_of(b); a.tri_a = TRI_LOWER;
        a.b = at(b, o + s1, o); a.b_rs = cs_of(b); a.b_ks = rs_of(b);
        a.c = x; a.c_rs = 1; a.c_cs = s2;
        a.m = s2; a.n = s1; a.k = s2; a.stop = p->d_info + b;
        p1.push_back(a);
        GemmProblem<T> c = problem<T>();   // T21 = -X T11^-1
        c.a = x; c.a_rs = 1; c.a_ks = s2;
        c.b = at(b, o, o); c.b_rs = cs_of(b); c.b_ks = rs_of(b); c.tri_b = TRI_UPPER;
        c.c = at(b, o + s1, o); c.c_rs = rs_of(b); c.c_cs = cs_of(b);
        c.alpha = minus_one; c.m = s2; c.n = s1; c.k = s1; c.stop = p->d_info + b;
        p2.push_back(c);
      }
    }
    CUCHOL_CHECK_CU(launch_list<T>(h, p1, p, s));
    CUCHOL_CHECK_CU(launch_list<T>(h, p2, p, s));
  }

  // ---- inverse: LAUUM, L^H L into workspace, then its lower triangle back ----
  std::vector<GemmProblem<T>> la, back;
  for (int b = 0; b < B; ++b) {
    const int nn = sh.n[b];
    T* wk = work + woff[b];
    GemmProblem<T> q = problem<T>();
    q.a = sh.a[b]; q.a_rs = cs_of(b); q.a_ks = rs_of(b); q.conj_a = 1; q.tri_a = TRI_UPPER;
    q.b = sh.a[b]; q.b_rs = cs_of(b); q.b_ks = rs_of(b); q.tri_b = TRI_UPPER;
    q.c = wk; q.c_rs = 1; q.c_cs = nn;
    q.m = nn; q.n = nn; q.k = nn; q.lower_only = 1; q.real_diag = 1; q.stop = p->d_info + b;
    la.push_back(q);
    GemmProblem<T> r = problem<T>();     // A := 0 * (nothing) + 1 * workspace (k = 0)
    r.a = wk; r.a_rs = 1; r.a_ks = nn; r.b = wk; r.b_rs = 1; r.b_ks = nn;
    r.c = sh.a[b]; r.c_rs = rs_of(b); r.c_cs = cs_of(b);
    r.cin = wk; r.cin_rs = 1; r.cin_cs = nn; r.beta = one;
    r.m = nn; r.n = nn; r.k = 0; r.lower_only = 1; r.stop = p->d_info + b;
    back.push_back(r);
  }
  CUCHOL_CHECK_CU(launch_list<T>(h, la, p, s));
  CUCHOL_CHECK_CU(launch_list<T>(h, back, p, s));
  return CUDA_SUCCESS;
}

}  // namespace

namespace {

void free_plan_memory(CUcholBatched p) {
  if (p->exec) cudaGraphExecDestroy(p->exec);
  if (p->graph) cudaGraphDestroy(p->graph);
  p->exec = nullptr;
  p->graph = nullptr;
  for (void* d : p->d_lists) cudaFree(d);
  p->d_lists.clear();
}

// Capture the batched sequence for `sh` with block size nb into p's graph.
template <typename T>
CUresult build_graph(CUcholBatched p, const BatchedShape<T>& sh, int nb) {
  free_plan_memory(p);
  cudaStream_t s = p->h->s_update;
  CUCHOL_CHECK(cudaStreamSynchronize(s));
  // pass 1: build and upload every problem list (no capture in progress)
  p->dry = true;
  p->reuse = false;
  CUresult rc = record_batched<T>(p, sh, nb, s);
  p->dry = false;
  if (rc != CUDA_SUCCESS) return rc;
  // pass 2: capture the launches, reusing the uploaded lists in the same order
  p->reuse = true;
  p->cursor = 0;
  CUCHOL_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  rc = record_batched<T>(p, sh, nb, s);
  p->reuse = false;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc != CUDA_SUCCESS) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  CUCHOL_CHECK(e);
  p->graph = g;
  CUCHOL_CHECK(cudaGraphInstantiate(&p->exec, g, 0));
  p->nb = nb;
  return CUDA_SUCCESS;
}

// Matrix b (blockIdx.x) of a packed batch := identity (column-major, ld n[b]).
template <typename T>
__global__ void set_identity_kernel(T* a, const long long* __restrict__ off, const int* __restrict__ n) {
  const int b = blockIdx.x;
  T* m = a + off[b];
  const long long nn = n[b];
  for (long long e = threadIdx.x; e < nn * nn; e += blockDim.x) {
    const long long r = e % nn, c = e / nn;
    m[e] = (r == c) ? from_real<T>(RealOf<T>(1)) : zero<T>();
  }
}

// Autotuner: time each candidate block size on an identity batch of the same shapes
// (the kernels do the same work for any SPD input) and keep the fastest.
template <typename T>
CUresult tune_nb(CUcholBatched p, const BatchedShape<T>& sh, int* best_nb) {
  // candidates: the grouped graphs with nb = 32 and 64, and (FP64) the persistent
  // kernel, written nb = -1 here
  std::vector<int> candidates = {32, 64};
  if (std::is_same<T, double>::value) candidates.push_back(-1);
  std::vector<long long> off(sh.batch);
  long long total = 0;
  for (int b = 0; b < sh.batch; ++b) { off[b] = total; total += (long long)sh.n[b] * sh.n[b]; }
  // everything acquired here is released by `res` on every return path
  struct Resources {
    T* scratch = nullptr;
    long long* d_off = nullptr;
    int* d_n = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Resources() {
      if (e0 != nullptr) cudaEventDestroy(e0);
      if (e1 != nullptr) cudaEventDestroy(e1);
      cudaFree(scratch);
      cudaFree(d_off);
      cudaFree(d_n);
    }
  } res;
  CUCHOL_CHECK(dev_malloc(&res.scratch, sizeof(T) * std::max<long long>(total, 1)));
  CUCHOL_CHECK(dev_malloc(&res.d_off, sizeof(long long) * sh.batch));
  CUCHOL_CHECK(dev_malloc(&res.d_n, sizeof(int) * sh.batch));
  CUCHOL_CHECK(cudaMemcpy(res.d_off, off.data(), sizeof(long long) * sh.batch, cudaMemcpyHostToDevice));
  CUCHOL_CHECK(cudaMemcpy(res.d_n, sh.n.data(), sizeof(int) * sh.batch, cudaMemcpyHostToDevice));
  T* scratch = res.scratch;
  long long* d_off = res.d_off;
  int* d_n = res.d_n;
  BatchedShape<T> id = sh;
  id.upper = false;
  for (int b = 0; b < sh.batch; ++b) { id.a[b] = scratch + off[b]; id.lda[b] = sh.n[b]; }
  float best = 1e30f;
  *best_nb = kBatchedMaxNb;
  cudaStream_t s = p->h->s_update;
  CUCHOL_CHECK(cudaEventCreate(&res.e0));
  CUCHOL_CHECK(cudaEventCreate(&res.e1));
  cudaEvent_t e0 = res.e0, e1 = res.e1;
  CUresult rc = CUDA_SUCCESS;
  for (int nb : candidates) {
    p->persistent = (nb < 0);
    rc = build_graph<T>(p, id, nb < 0 ? kBatchedMaxNb : nb);
    if (rc != CUDA_SUCCESS) break;
    float ms_min = 1e30f;
    for (int rep = 0; rep < 3; ++rep) {
      set_identity_kernel<T><<<sh.batch, 256, 0, s>>>(scratch, d_off, d_n);
      cudaEventRecord(e0, s);
      cudaGraphLaunch(p->exec, s);
      cudaEventRecord(e1, s);
      if (cudaEventSynchronize(e1) != cudaSuccess) { rc = CUDA_ERROR_UNKNOWN; break; }
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      ms_min = std::min(ms_min, ms);
    }
    if (rc != CUDA_SUCCESS) break;
    if (ms_min < best) { best = ms_min; *best_nb = nb; }
  }
  free_plan_memory(p);
  return rc;
}

}  // namespace

namespace {

template <typename T>
CUresult batched_create(CUcholBatched* out, CULAPACKhandle h, char type, CBlasUplo uplo, int batch,
                        const int* n, const CUdeviceptr* A, const int* lda, int flags, int nb) {
  // nb: 0 = tuned, 8..64 (multiple of 8) = the grouped graph with that block size,
  // -1 = the persistent kernel (FP64 only)
  const bool nb_ok = (nb == -1 && std::is_same<T, double>::value) ||
                     (nb >= 0 && nb <= kBatchedMaxNb && (nb == 0 || nb % 8 == 0));
  if (out == nullptr || h == nullptr || batch <= 0 || n == nullptr || A == nullptr || lda == nullptr ||
      (uplo != CBlasLower && uplo != CBlasUpper) || !nb_ok)
    return CUDA_ERROR_INVALID_VALUE;
  BatchedShape<T> sh;
  sh.upper = (uplo == CBlasUpper);
  sh.batch = batch;
  sh.flags = flags | 1;
  size_t work = 1;
  for (int b = 0; b < batch; ++b) {
    if (n[b] < 1 || lda[b] < n[b]) {
      if (xerbla != nullptr) xerbla(type == 'D' ? "cuDcholBatchedCreate" : "cuScholBatchedCreate", 4);
      return CUDA_ERROR_INVALID_VALUE;
    }
    sh.n.push_back(n[b]);
    sh.a.push_back(reinterpret_cast<T*>(A[b]));
    sh.lda.push_back(lda[b]);
    if (flags & 4) work += (size_t)n[b] * n[b];   // the inverse's workspace
  }
  auto* p = new (std::nothrow) __cucholbatched_st;
  if (p == nullptr) return CUDA_ERROR_OUT_OF_MEMORY;
  p->h = h;
  p->type = type;
  p->batch = batch;
  p->nb = 0;
  p->d_info = nullptr;
  p->d_logdet = nullptr;
  p->d_w = nullptr;
  p->d_work = nullptr;
  p->graph = nullptr;
  p->exec = nullptr;
  p->persistent = 0;
  p->d_next = nullptr;
  p->d_wp = nullptr;
  p->wp_tiles = 1;
  p->dry = false;
  p->reuse = false;
  p->cursor = 0;
  CUresult rc = CUDA_SUCCESS;
  auto fail = [&](CUresult r) {
    free_plan_memory(p);
    cudaFree(p->d_info); cudaFree(p->d_logdet); cudaFree(p->d_w); cudaFree(p->d_work);
    cudaFree(p->d_next); cudaFree(p->d_wp);
    delete p;
    return r;
  };
  using Smem = DiagSmem<T, kBatchedMaxNb>;
  if (cudaFuncSetAttribute(diag_factor_batched_kernel<T, kBatchedMaxNb, kDiagThreads2>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Smem::bytes) != cudaSuccess ||
      cudaFuncSetAttribute(diag_invert_batched_kernel<T, kBatchedMaxNb, kDiagThreads2>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Smem::bytes) != cudaSuccess ||
      dev_malloc(&p->d_info, sizeof(int) * batch) != cudaSuccess ||
      dev_malloc(&p->d_logdet, sizeof(double) * batch) != cudaSuccess ||
      dev_malloc(&p->d_w, sizeof(T) * (size_t)batch * kBatchedMaxNb * kBatchedMaxNb) != cudaSuccess ||
      dev_malloc(&p->d_work, sizeof(T) * std::max<size_t>(work, 1)) != cudaSuccess)
    return fail(report(cudaGetLastError(), "cudaMalloc", __func__, __FILE__, __LINE__));
  int nmax = 1;
  for (int b = 0; b < batch; ++b) nmax = std::max(nmax, n[b]);
  p->wp_tiles = (nmax + kBatchedMaxNb - 1) / kBatchedMaxNb;
  if (std::is_same<T, double>::value &&
      (dev_malloc(&p->d_next, sizeof(int)) != cudaSuccess ||
       dev_malloc(&p->d_wp, sizeof(double) * (size_t)h->num_sms * p->wp_tiles * kBatchedMaxNb * kBatchedMaxNb) !=
           cudaSuccess))
    return fail(report(cudaGetLastError(), "cudaMalloc", __func__, __FILE__, __LINE__));
  if (nb == 0) {
    rc = tune_nb<T>(p, sh, &nb);
    if (rc != CUDA_SUCCESS) return fail(rc);
  }
  p->persistent = (nb < 0);
  rc = build_graph<T>(p, sh, nb < 0 ? kBatchedMaxNb : nb);
  if (rc != CUDA_SUCCESS) return fail(rc);
  *out = p;
  return CUDA_SUCCESS;
}

}  // namespace

extern "C" CUCHOL_EXPORT CUresult cuDcholBatchedCreate(CUcholBatched* plan, CULAPACKhandle h, CBlasUplo uplo,
                                                       int batch, const int* n, const CUdeviceptr* A,
                                                       const int* lda, int flags, int nb) {
  return batched_create<double>(plan, h, 'D', uplo, batch, n, A, lda, flags, nb);
}

extern "C" CUCHOL_EXPORT CUresult cuScholBatchedCreate(CUcholBatched* plan, CULAPACKhandle h, CBlasUplo uplo,
                                                       int batch, const int* n, const CUdeviceptr* A,
                                                       const int* lda, int flags, int nb) {
  return batched_create<float>(plan, h, 'S', uplo, batch, n, A, lda, flags, nb);
}

extern "C" CUCHOL_EXPORT CUresult cuCholBatchedRun(CUcholBatched p, CUstream stream) {
  if (p == nullptr || p->exec == nullptr) return CUDA_ERROR_INVALID_VALUE;
  CUCHOL_CHECK(cudaGraphLaunch(p->exec, reinterpret_cast<cudaStream_t>(stream)));
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuCholBatchedResults(CUcholBatched p, long* info, double* logdet) {
  if (p == nullptr) return CUDA_ERROR_INVALID_VALUE;
  CUCHOL_CHECK(cudaDeviceSynchronize());
  if (info != nullptr) {
    std::vector<int> tmp(p->batch);
    CUCHOL_CHECK(cudaMemcpy(tmp.data(), p->d_info, sizeof(int) * p->batch, cudaMemcpyDeviceToHost));
    for (int b = 0; b < p->batch; ++b) info[b] = tmp[b];
  }
  if (logdet != nullptr)
    CUCHOL_CHECK(cudaMemcpy(logdet, p->d_logdet, sizeof(double) * p->batch, cudaMemcpyDeviceToHost));
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuCholBatchedGetBlockSize(CUcholBatched p, int* nb) {
  if (p == nullptr || nb == nullptr) return CUDA_ERROR_INVALID_VALUE;
  *nb = p->persistent ? -1 : p->nb;
  return CUDA_SUCCESS;
}

extern "C" CUCHOL_EXPORT CUresult cuCholBatchedDestroy(CUcholBatched p) {
  if (p == nullptr) return CUDA_ERROR_INVALID_VALUE;
  cudaDeviceSynchronize();
  free_plan_memory(p);
  cudaFree(p->d_info);
  cudaFree(p->d_logdet);
  cudaFree(p->d_w);
  cudaFree(p->d_work);
  cudaFree(p->d_next);
  cudaFree(p->d_wp);
  delete p;
  return CUDA_SUCCESS;
}
