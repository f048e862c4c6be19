// Persistent form of the batched FP64 plan (included at the end of lapack.cu, after
// batched.cuh): one launch factors, log-dets and inverts every matrix of the batch.
//
// Each CTA (one per SM) takes whole matrices from a work queue ordered by size,
// largest first (the longest-processing-time rule: the last matrices taken are the
// cheapest, so the CTAs finish together), and runs the blocked algorithms on the
// matrix in place as a sequence of phases over 64 x 64 tiles:
//   ?potrf  for each block column k: the diagonal block factored (and its inverse W
//           formed) in shared memory; panel tiles L_ik = A_ik W^T; trailing tiles
//           A_ij -= L_ik L_jk^T (lower part of the diagonal tiles only);
//   ?trtri  every diagonal tile replaced by the inverse that the factor formed for its
//           panel (kept aside until the factor has succeeded); then, block column j from the last
//           to the first, X_ij = sum_{l=j+1..i} inv(L)_il L_lj (rows from the bottom
//           up, so each row still reads the L_lj of the rows above it) and then
//           inv(L)_ij = -X_ij inv(L_jj);
//   ?lauum  C_ij = sum_{l >= i} inv(L)_li^T inv(L)_lj, block column j from the first,
//           rows from the top down: each tile reads only tiles that are rewritten
//           after it.
// The jobs of a phase are independent of each other (by the orders above), so the
// operand tiles of the next job are fetched (cp.async, two-stage ring) while the
// current one runs on the FP64 tensor cores (mma.sync m16n8k4, eight warps of
// 32 x 16 outputs); phases are separated by barriers.  The diagonal steps reuse the
// one-CTA kernels' bodies (diag_factor_block, diag_invert_block).  A matrix whose
// factor fails keeps its info word and is left as the factor left it.
#pragma once

namespace {
namespace bpk {

constexpr int NB = 64, THREADS = 256, LDS = 68;      // tile order; staged rows padded to 68
constexpr int TILE = NB * LDS;                        // doubles per staged operand tile
constexpr size_t RING_BYTES = 2 * 2 * TILE * sizeof(double);   // 2 stages x (A, B)

struct MatDesc {
  double* a;
  int n, lda;
  int* info;
  double* logdet;     // or null
};

// Operand of a tile product: element (r, k) at p[r * rs + k * ks] for r < m, k < kk;
// tri: TRI_LOWER keeps k <= r, TRI_UPPER keeps k >= r (the rest reads as zero).
struct Opnd {
  const double* p;
  long long rs, ks;
  int m, kk, tri;
};

// Output of a job: C(r, c) at p[r * rs + c * cs], r < m, c < n;
// C := alpha * acc + beta * C, lower: only r >= c.
struct Out {
  double* p;
  long long rs, cs;
  int m, n;
  double alpha, beta;
  int lower;
};

__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Stage one operand tile into X[k * LDS + r] (cp.async, zeros where not kept).  Rows
// contiguous in memory: consecutive lanes take consecutive rows (conflict-free
// shared stores).  k contiguous: each 8 lanes take 8 consecutive k (64 contiguous
// bytes) of one row, 4 rows per warp, so the shared stores, 68 doubles apart along
// k, spread over the banks.
__device__ __forceinline__ void stage(const Opnd& o, double* X) {
  for (int e = threadIdx.x; e < NB * NB; e += THREADS) {
    int r, k;
    if (o.rs == 1) { r = e & (NB - 1); k = e >> 6; }
    else { k = (e & 7) | (((e >> 9) & 7) << 3); r = (e >> 3) & (NB - 1); }
    const bool v = r < o.m && k < o.kk && (o.tri == TRI_NONE || (o.tri == TRI_LOWER ? k <= r : k >= r));
    cp_async_elem<double>(&X[k * LDS + r], v ? o.p + r * o.rs + k * o.ks : o.p, v);
  }
}

// acc += A B^T for the staged tiles (k = 0..63).  Warp w: rows 32 (w & 1) .. + 31,
// columns 16 (w >> 1) .. + 15; fragment (g, t) of lane = 4 g + t.
__device__ __forceinline__ void tile_mma(double (&acc)[2][2][4], const double* As, const double* Bs) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = (warp & 1) * 32, c0 = (warp >> 1) * 16;
#pragma unroll 4
  for (int k4 = 0; k4 < NB; k4 += 4) {
    const double* a = As + (k4 + t) * LDS + r0 + g;
    const double* b = Bs + (k4 + t) * LDS + c0 + g;
    const double a00 = a[0], a01 = a[8], a10 = a[16], a11 = a[24];
    const double b0 = b[0], b1 = b[8];
    cuchol::dmma_m16n8k4(acc[0][0], a00, a01, b0);
    cuchol::dmma_m16n8k4(acc[0][1], a00, a01, b1);
    cuchol::dmma_m16n8k4(acc[1][0], a10, a11, b0);
    cuchol::dmma_m16n8k4(acc[1][1], a10, a11, b1);
  }
}

__device__ __forceinline__ void store_out(const double (&acc)[2][2][4], const Out& o) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  const int r0 = (warp & 1) * 32, c0 = (warp >> 1) * 16;
#pragma unroll
  for (int mb = 0; mb < 2; ++mb)
#pragma unroll
    for (int nb8 = 0; nb8 < 2; ++nb8)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int r = r0 + mb * 16 + g + (e >> 1) * 8, c = c0 + nb8 * 8 + 2 * t + (e & 1);
        if (r < o.m && c < o.n && (!o.lower || r >= c)) {
          double* q = o.p + r * o.rs + c * o.cs;
          double v = o.alpha * acc[mb][nb8][e];
          if (o.beta != 0.0) v = fma(o.beta, *q, v);
          *q = v;
        }
      }
}

// Runs the njobs jobs of one phase: job j has nterms(j) terms term(j, t, &a, &b) and
// output out(j).  Term loads run one item ahead, across job boundaries.
template <typename NT, typename TF, typename OF>
__device__ void run_phase(int njobs, NT nterms, TF term, OF out, double* ring) {
  if (njobs <= 0) return;
  double acc[2][2][4];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;
  auto issue = [&](int j, int t, int st) {
    Opnd A, B;
    term(j, t, A, B);
    stage(A, ring + st * 2 * TILE);
    stage(B, ring + st * 2 * TILE + TILE);
  };
  int job = 0, tt = 0, st = 0, jn = nterms(0);
  issue(0, 0, 0);
  cp_commit();
  while (true) {
    int nj = job, nt = tt + 1;
    if (nt >= jn) { nj = job + 1; nt = 0; }
    const bool more = nj < njobs;
    if (more) issue(nj, nt, st ^ 1);
    cp_commit();
    cp_wait1();
    __syncthreads();
    tile_mma(acc, ring + st * 2 * TILE, ring + st * 2 * TILE + TILE);
    __syncthreads();                                 // stage st is refilled next
    if (tt == jn - 1) {
      store_out(acc, out(job));
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.0;
    }
    if (!more) break;
    if (nj != job) jn = nterms(nj);
    job = nj;
    tt = nt;
    st ^= 1;
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();                                   // outputs visible to the next phase
}

// Factor, log det and inverse of one matrix (lower view A(i, j) = a[i * rs + j * cs]).
__device__ void process(const MatDesc& M, long long rs, long long cs, bool inverse, double* W, double* ring) {
  const int n = M.n, nt = (n + NB - 1) / NB;
  double* a = M.a;
  auto tl = [&](int i, int j) { return a + (long long)i * NB * rs + (long long)j * NB * cs; };
  auto ext = [&](int i) { return min(NB, n - i * NB); };

  // W + k * NB * NB: the inverse of diagonal factor block k (ld NB), kept for the panel
  // below it and, with the inverse to follow, for ?trtri
  auto Wk = [&](int k) { return W + (inverse ? (size_t)k * NB * NB : 0); };

  // ---- ?potrf ----
  for (int k = 0; k < nt; ++k) {
    const int jb = ext(k);
    const bool below = (k + 1 < nt);
    cuchol::diag_factor_block<double, NB, THREADS>(tl(k, k), rs, cs, jb, (below || inverse) ? Wk(k) : nullptr,
                                                   NB, (long long)k * NB, M.info, M.logdet);
    __syncthreads();
    if (cuchol::cta_aborted(M.info)) return;         // this matrix's factor failed
    if (!below) break;
    const int m = nt - k - 1;
    // panel: L_ik = A_ik W^T, i = k+1 ..
    run_phase(
        m, [](int) { return 1; },
        [&](int j, int, Opnd& A, Opnd& B) {
          const int i = k + 1 + j;
          A = Opnd{tl(i, k), rs, cs, ext(i), jb, TRI_NONE};
          B = Opnd{Wk(k), 1, NB, jb, jb, TRI_NONE};    // B(c, kk) = W(c, kk): zeros above the diagonal
        },
        [&](int j) {
          const int i = k + 1 + j;
          return Out{tl(i, k), rs, cs, ext(i), jb, 1.0, 0.0, 0};
        },
        ring);
    // trailing: A_ij -= L_ik L_jk^T, k < j <= i (jobs in order j = k+1.., i = j..)
    run_phase(
        m * (m + 1) / 2, [](int) { return 1; },
        [&](int q, int, Opnd& A, Opnd& B) {
          int jj = 0;
          while (q >= m - jj) { q -= m - jj; ++jj; }
          const int j = k + 1 + jj, i = j + q;
          A = Opnd{tl(i, k), rs, cs, ext(i), jb, TRI_NONE};
          B = Opnd{tl(j, k), rs, cs, ext(j), jb, TRI_NONE};
        },
        [&](int q) {
          int jj = 0;
          while (q >= m - jj) { q -= m - jj; ++jj; }
          const int j = k + 1 + jj, i = j + q;
          return Out{tl(i, j), rs, cs, ext(i), ext(j), -1.0, 1.0, i == j};
        },
        ring);
  }
  if (!inverse) return;

  // ---- ?trtri: the diagonal tiles take the inverses formed by the factor, then the
  // block columns from the last ----
  for (int k = 0; k < nt; ++k) {
    const int jb = ext(k);
    const double* w = Wk(k);
    for (int e = threadIdx.x; e < jb * jb; e += THREADS) {
      const int r = e % jb, c = e / jb;
      if (r >= c) tl(k, k)[r * rs + c * cs] = w[r + c * NB];
    }
  }
  __syncthreads();
  for (int j = nt - 2; j >= 0; --j) {
    const int m = nt - j - 1;
    // X_ij = sum_{l = j+1 .. i} inv(L)_il L_lj, rows i from the bottom up (in place)
    run_phase(
        m, [&](int q) { return m - q; },              // row i = nt-1-q has i - j terms
        [&](int q, int t, Opnd& A, Opnd& B) {
          const int i = nt - 1 - q, l = j + 1 + t;
          // A(r, kk) = inv(L)_il(r, kk); the diagonal tile is lower triangular
          A = Opnd{tl(i, l), rs, cs, ext(i), ext(l), l == i ? TRI_LOWER : TRI_NONE};
          // B(c, kk) = L_lj(kk, c): the transposed view
          B = Opnd{tl(l, j), cs, rs, ext(j), ext(l), TRI_NONE};
        },
        [&](int q) {
          const int i = nt - 1 - q;
          return Out{tl(i, j), rs, cs, ext(i), ext(j), 1.0, 0.0, 0};
        },
        ring);
    // inv(L)_ij = -X_ij inv(L_jj): B(c, kk) = inv(L_jj)(kk, c), nonzero for kk >= c
    run_phase(
        m, [](int) { return 1; },
        [&](int q, int, Opnd& A, Opnd& B) {
          const int i = j + 1 + q;
          A = Opnd{tl(i, j), rs, cs, ext(i), ext(j), TRI_NONE};
          B = Opnd{tl(j, j), cs, rs, ext(j), ext(j), TRI_UPPER};
        },
        [&](int q) {
          const int i = j + 1 + q;
          return Out{tl(i, j), rs, cs, ext(i), ext(j), -1.0, 0.0, 0};
        },
        ring);
  }
  // ---- ?lauum: C_ij = sum_{l >= i} inv(L)_li^T inv(L)_lj, j ascending, i ascending ----
  run_phase(
      nt * (nt + 1) / 2,
      [&](int q) {
        int j = 0;
        while (q >= nt - j) { q -= nt - j; ++j; }
        const int i = j + q;
        return nt - i;
      },
      [&](int q, int t, Opnd& A, Opnd& B) {
        int j = 0;
        while (q >= nt - j) { q -= nt - j; ++j; }
        const int i = j + q, l = i + t;
        // A(r, kk) = inv(L)_li(kk, r) (transposed view; the diagonal tile l == i is
        // lower triangular: kk >= r), B(c, kk) = inv(L)_lj(kk, c) (lower when l == j)
        A = Opnd{tl(l, i), cs, rs, ext(i), ext(l), l == i ? TRI_UPPER : TRI_NONE};
        B = Opnd{tl(l, j), cs, rs, ext(j), ext(l), l == j ? TRI_UPPER : TRI_NONE};
      },
      [&](int q) {
        int j = 0;
        while (q >= nt - j) { q -= nt - j; ++j; }
        const int i = j + q;
        return Out{tl(i, j), rs, cs, ext(i), ext(j), 1.0, 0.0, i == j};
      },
      ring);
}

// order: matrix indices, largest first; *next: the queue head (zero at launch).
// wbuf: per CTA, ntmax inverse blocks of NB x NB (ntmax = block columns of the largest
// matrix).
__global__ void __launch_bounds__(THREADS, 1)
    persistent_kernel(const MatDesc* __restrict__ mats, const int* __restrict__ order, int batch, int* next,
                      int upper, int inverse, double* wbuf, int ntmax) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* ring = reinterpret_cast<double*>(smem_raw);
  double* W = wbuf + (size_t)blockIdx.x * ntmax * NB * NB;
  __shared__ int s_w;
  while (true) {
    if (threadIdx.x == 0) s_w = atomicAdd(next, 1);
    __syncthreads();
    const int w = s_w;
    __syncthreads();
    if (w >= batch) break;
    const MatDesc M = mats[order[w]];
    const long long rs = upper ? M.lda : 1, cs = upper ? 1 : M.lda;
    process(M, rs, cs, inverse != 0, W, ring);
    __syncthreads();
  }
}

constexpr size_t smem_bytes() {
  return RING_BYTES > cuchol::DiagSmem<double, NB>::bytes ? RING_BYTES : cuchol::DiagSmem<double, NB>::bytes;
}

}  // namespace bpk
}  // namespace

namespace {

// The persistent form as the plan's recorded sequence: per-matrix descriptors and
// the size order uploaded once; per run, the result words and the queue head
// cleared, then one launch (one CTA per SM).
template <typename T>
CUresult record_persistent(CUcholBatched p, const BatchedShape<T>& sh, cudaStream_t s) {
  static_assert(std::is_same<T, double>::value, "the persistent form is FP64");
  CULAPACKhandle h = p->h;
  const int B = sh.batch;
  std::vector<bpk::MatDesc> mats(B);
  for (int b = 0; b < B; ++b)
    mats[b] = bpk::MatDesc{sh.a[b], sh.n[b], (int)sh.lda[b], p->d_info + b,
                           (sh.flags & 2) ? p->d_logdet + b : nullptr};
  std::vector<int> order(B);
  for (int b = 0; b < B; ++b) order[b] = b;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return sh.n[x] > sh.n[y]; });
  CUresult rc = CUDA_SUCCESS;
  const bpk::MatDesc* dm = upload(p, mats, &rc);
  if (dm == nullptr) return rc == CUDA_SUCCESS ? CUDA_ERROR_OUT_OF_MEMORY : rc;
  const int* dord = upload(p, order, &rc);
  if (dord == nullptr) return rc == CUDA_SUCCESS ? CUDA_ERROR_OUT_OF_MEMORY : rc;
  if (p->dry) return CUDA_SUCCESS;
  static bool attr = false;
  if (!attr) {
    CUCHOL_CHECK(cudaFuncSetAttribute(bpk::persistent_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)bpk::smem_bytes()));
    attr = true;
  }
  CUCHOL_CHECK(cudaMemsetAsync(p->d_info, 0, sizeof(int) * B, s));
  CUCHOL_CHECK(cudaMemsetAsync(p->d_logdet, 0, sizeof(double) * B, s));
  CUCHOL_CHECK(cudaMemsetAsync(p->d_next, 0, sizeof(int), s));
  const int grid = std::min(B, h->num_sms);
  bpk::persistent_kernel<<<grid, bpk::THREADS, bpk::smem_bytes(), s>>>(dm, dord, B, p->d_next, sh.upper ? 1 : 0,
                                                                         (sh.flags & 4) ? 1 : 0, p->d_wp,
                                                                         p->wp_tiles);
  ++h->launches;
  CUCHOL_CHECK(cudaGetLastError());
  return CUDA_SUCCESS;
}

}  // namespace
