// Batched Dyson solve per (q, iW): products, FP64 Cholesky, log-determinant, W.
#include <algorithm>
#include <string>

#include "chol.cuh"
#include "dyson.cuh"
#include "kernels.cuh"
#include "tc_gemm.cuh"
#include "zgemm.cuh"

namespace cq {

__global__ void k_zero_upper_adjoint(double2* __restrict__ L, double2* __restrict__ LH, int64_t Np,
                                     int64_t total) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = idx / (Np * Np), e = idx % (Np * Np);
    const int64_t i = e / Np, j = e % Np;
    double2* Lb = L + b * Np * Np;
    // LH[i][j] = conj(L[j][i]) for j >= i (lower element of L), 0 otherwise
    double2 v = make_double2(0, 0);
    if (j >= i) {
      const double2 l = Lb[j * Np + i];
      v = make_double2(l.x, -l.y);
    }
    LH[idx] = v;
    if (j > i) Lb[i * Np + j] = make_double2(0, 0);
  }
}

// E = DH + DH^H + F with only the lower triangle (i >= j) of the Hermitian F computed: one CTA
// per lower pair of 32 x 32 tiles (E is Hermitian), problem blockIdx.y.
__global__ void __launch_bounds__(256) k_herm_sum(const float2* __restrict__ DH,
                                                  const float2* __restrict__ F,
                                                  float2* __restrict__ E, int64_t Np) {
  int I, J;
  tile_pair((int)blockIdx.x, I, J);
  const int64_t off = (int64_t)blockIdx.y * Np * Np;
  herm_sum_pair(DH + off, F + off, E + off, Np, I, J);
}

// Hermitian completion: A[i][j] = conj(A[j][i]) for j > i (32 x 32 tiles on or above the
// diagonal, the lower tile read through shared memory); complex64 or complex128
template <typename C>
__global__ void k_mirror_upper(C* __restrict__ A, int64_t n, int64_t stride) {
  __shared__ C tile[32][33];
  const int64_t i0 = (int64_t)blockIdx.y * 32, j0 = (int64_t)blockIdx.x * 32;
  if (j0 < i0) return;
  C* a = A + (int64_t)blockIdx.z * stride;
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {  // lower tile (j0.., i0..)
    const int64_t r = j0 + ty, c = i0 + threadIdx.x;
    tile[ty][threadIdx.x] = (r < n && c < n) ? a[r * n + c] : mk<C>(0.0, 0.0);
  }
  __syncthreads();
  for (int ty = threadIdx.y; ty < 32; ty += blockDim.y) {
    const int64_t i = i0 + ty, j = j0 + threadIdx.x;
    if (i < n && j < n && j > i) {
      const C v = tile[threadIdx.x][ty];  // A[j][i]
      a[i * n + j] = mk<C>(v.x, -v.y);
    }
  }
}

template <typename C>
void mirror_upper(C* A, int64_t n, int64_t nbatch, cudaStream_t s, int64_t stride) {
  CQ_REQUIRE(nbatch <= 65535, COQUI_B200_EINVAL, "mirror: too many problems per launch");
  const unsigned t = (unsigned)((n + 31) / 32);
  k_mirror_upper<C><<<dim3(t, t, (unsigned)nbatch), dim3(32, 8), 0, s>>>(A, n, stride > 0 ? stride : n * n);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

void launch_mirror_upper(float2* A, int64_t n, int64_t nbatch, cudaStream_t s, int64_t stride) {
  mirror_upper<float2>(A, n, nbatch, s, stride);
}

// FP64 form: E = Z + Z^H + F (Hermitian, written whole) with Z = D^H upper triangular and F
// Hermitian with only its lower triangle formed
__global__ void k_herm_sum_c128(const double2* __restrict__ Z, const double2* __restrict__ F,
                                double2* __restrict__ E, int64_t n, int64_t total) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / (n * n), e = i % (n * n), r = e / n, c = e % n;
    const int64_t t = b * n * n + c * n + r;  // the transposed element
    const double2 z = Z[i], zt = Z[t];
    const double2 f = r >= c ? F[i] : make_double2(F[t].x, -F[t].y);
    E[i] = make_double2(z.x + zt.x + f.x, z.y - zt.y + f.y);
  }
}


void launch_zero_upper_and_adjoint(double2* L, double2* LH, int64_t Np, int64_t nbatch,
                                   cudaStream_t s) {
  const int64_t total = Np * Np * nbatch;
  k_zero_upper_adjoint<<<grid_for(total, 256), 256, 0, s>>>(L, LH, Np, total);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
}

// The factorisation keeps each 32 x 32 diagonal block of its factor in shared memory only
// (global memory gets the panel blocks below it and, in the upper triangle, the block's
// inverse adjoint).  This kernel forms the diagonal blocks again the way the factorisation
// does: C_jj = chol(A_jj - sum_{kb < j} L_j,kb L_j,kb^H) from I - M = A and the stored panel
// blocks, and writes them into A's lower triangle.  One CTA per (block j, problem).
constexpr int kDiagB = 32;
__global__ void __launch_bounds__(256) k_chol_diag_blocks(const double2* __restrict__ Mall,
                                                          double2* __restrict__ Aall, int64_t n,
                                                          int* __restrict__ info) {
  __shared__ double2 S[kDiagB][kDiagB + 1];
  __shared__ double2 T[kDiagB][kDiagB + 1];
  const int64_t p = blockIdx.y, j0 = (int64_t)blockIdx.x * kDiagB;
  const int jb = (int)((n - j0) < kDiagB ? (n - j0) : kDiagB);
  const double2* M = Mall + p * n * n;
  double2* A = Aall + p * n * n;
  for (int i = threadIdx.x; i < kDiagB * kDiagB; i += blockDim.x) {
    const int r = i / kDiagB, c = i % kDiagB;
    double2 v = make_double2(0.0, 0.0);
    if (r < jb && c <= r) {
      const double2 m = M[(j0 + r) * n + j0 + c];
      v = make_double2((r == c ? 1.0 : 0.0) - m.x, -m.y);
    }
    S[r][c] = v;
  }
  for (int64_t k0 = 0; k0 < j0; k0 += kDiagB) {  // panel blocks to the left are whole blocks
    __syncthreads();
    for (int i = threadIdx.x; i < kDiagB * kDiagB; i += blockDim.x) {
      const int r = i / kDiagB, c = i % kDiagB;
      T[r][c] = r < jb ? A[(j0 + r) * n + k0 + c] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kDiagB * kDiagB; i += blockDim.x) {
      const int r = i / kDiagB, c = i % kDiagB;
      if (r >= jb || c > r) continue;
      double sr = 0.0, si = 0.0;
      for (int k = 0; k < kDiagB; ++k) {  // T[r][k] conj(T[c][k])
        const double2 a = T[r][k], b = T[c][k];
        sr += a.x * b.x + a.y * b.y;
        si += a.y * b.x - a.x * b.y;
      }
      S[r][c].x -= sr;
      S[r][c].y -= si;
    }
  }
  for (int q = 0; q < jb; ++q) {  // right-looking factorisation of the 32 x 32 block
    __syncthreads();
    const double d2 = S[q][q].x;
    const double d = d2 > 0.0 ? sqrt(d2) : 0.0;
    if (!(d2 > 0.0) && threadIdx.x == 0) info[p] = 1;
    const double inv = d > 0.0 ? 1.0 / d : 0.0;
    __syncthreads();
    if (threadIdx.x == 0) S[q][q] = make_double2(d, 0.0);
    for (int r = q + 1 + threadIdx.x; r < jb; r += blockDim.x) {
      S[r][q].x *= inv;
      S[r][q].y *= inv;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kDiagB * kDiagB; i += blockDim.x) {
      const int r = i / kDiagB, c = i % kDiagB;
      if (r >= jb || c <= q || c > r) continue;
      const double2 a = S[r][q], b = S[c][q];  // S[r][c] -= a conj(b)
      S[r][c].x -= a.x * b.x + a.y * b.y;
      S[r][c].y -= a.y * b.x - a.x * b.y;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kDiagB * kDiagB; i += blockDim.x) {
    const int r = i / kDiagB, c = i % kDiagB;
    if (r < jb && c <= r) A[(j0 + r) * n + j0 + c] = S[r][c];
  }
}

// A = L L^H for nbatch Hermitian matrices on the library's FP64 factorisation: it factors
// I - M, so M = I - A goes in; the panel blocks of L land in A's lower triangle, the diagonal
// blocks are formed again from them (k_chol_diag_blocks), and the strict upper triangle is
// left as workspace.  The first nonzero per-problem status (a pivot that was not positive) is
// returned.
int cholesky_lower_batched(double2* A, int64_t Np, int64_t nbatch, cudaStream_t s) {
  DevBuf<double2> M, tr;
  DevBuf<double> ld;
  DevBuf<int> dinfo;
  M.ensure((size_t)nbatch * Np * Np);
  tr.ensure(nbatch);
  ld.ensure(nbatch);
  dinfo.ensure(nbatch);
  launch_eye_minus<double>(A, M.p, Np, nbatch, s);
  launch_chol_inv_c128(M.p, A, ld.p, tr.p, dinfo.p, Np, nbatch, s);
  const int64_t nblk = (Np + kDiagB - 1) / kDiagB;
  CQ_REQUIRE(nblk <= 65535 && nbatch <= 65535, COQUI_B200_EUNSUPPORTED,
             "Cholesky of V: too many blocks or matrices");
  k_chol_diag_blocks<<<dim3((unsigned)nblk, (unsigned)nbatch), 256, 0, s>>>(M.p, A, Np, dinfo.p);
  count_launch();
  CQ_CHECK_CUDA(cudaGetLastError());
  std::vector<int> info(nbatch);
  CQ_CHECK_CUDA(cudaMemcpyAsync(info.data(), dinfo.p, nbatch * sizeof(int), cudaMemcpyDeviceToHost, s));
  CQ_CHECK_CUDA(cudaStreamSynchronize(s));
  for (int v : info)
    if (v != 0) return v;
  return 0;
}

namespace {
// The mixed form with the tensor-core inverse keeps M, the inverse levels' scratch and E in
// the chunk's own Pi(iW) slices (dead once P1 = L^H Pi is formed; W overwrites them last).
bool m_in_pi(int64_t Np, bool mixed, bool want_w) { return mixed && want_w && Np > kInvGroup; }

// scratch bytes per problem: T1 (es), M (es, unless in Pi), A (c128), Y (c128; the mixed
// form's W operands)
size_t dyson_bytes_per_problem(int64_t Np, bool mixed, bool want_w) {
  const size_t NN = (size_t)Np * Np, es = mixed ? sizeof(float2) : sizeof(double2);
  return NN * (es + (m_in_pi(Np, mixed, want_w) ? 0 : es) + sizeof(double2) +
               (mixed && want_w ? sizeof(double2) : 0)) +
         64;
}
constexpr double kScratchShare = 0.6;  // of the free device memory, per chunk
}  // namespace

size_t dyson_reserve_bytes(int64_t Np, int64_t nprob, bool mixed) {
  const int64_t n = std::min<int64_t>(nprob, 2 * chol_wave_size());
  return (size_t)((double)(dyson_bytes_per_problem(Np, mixed, true) * (size_t)n + 1024) /
                  kScratchShare);
}

void dyson_run(const DysonArgs& a, DevBuf<unsigned char>& scratch, cudaStream_t s,
               std::vector<double>* logdet, std::vector<double2>* trace) {
  const int64_t Np = a.Np, NN = Np * Np, nq = a.nq, nw = a.nw;
  const size_t es = a.mixed ? sizeof(float2) : sizeof(double2);
  const bool mpi = m_in_pi(Np, a.mixed, a.want_w);
  const size_t per = dyson_bytes_per_problem(Np, a.mixed, a.want_w);
  // Chunks of the flattened (w, q) problem list (per-q operands addressed periodically), as
  // many problems per chunk as ~60% of the free device memory allows, so the factorisation
  // kernel sees whole waves of problems (one CTA per problem)
  size_t fr = 0, tot = 0;
  CQ_CHECK_CUDA(cudaMemGetInfo(&fr, &tot));
  size_t budget = std::max(scratch.n, (size_t)(kScratchShare * (double)(fr + scratch.n)));
  // while a graph is captured the scratch keeps its size (no device allocation or free inside
  // the capture) when it holds at least one problem
  if (a.keep_scratch && scratch.n >= per + 1024) budget = scratch.n - 1024;
  const int64_t nprob = nw * nq;
  int64_t nbq = std::max<int64_t>(1, std::min<int64_t>(nprob, (int64_t)(budget / per)));
  if (nbq < nprob) {
    // several chunks: whole waves of the one-CTA factorisation per chunk (a chunk of 1.5 waves
    // leaves half the GPU idle during its second wave)
    const int64_t wave = chol_wave_size();
    if (nbq >= wave) nbq = nbq / wave * wave;
  }
  scratch.ensure(per * nbq + 1024);
  unsigned char* base = scratch.p;
  auto carve = [&](size_t bytes) {
    unsigned char* p = base;
    base += (bytes + 255) & ~(size_t)255;
    return p;
  };
  unsigned char* T1 = carve(nbq * NN * es);
  unsigned char* Mb0 = mpi ? nullptr : carve(nbq * NN * es);
  double2* A = (double2*)carve(nbq * NN * sizeof(double2));
  double2* Y = a.mixed && a.want_w ? (double2*)carve(nbq * NN * sizeof(double2)) : nullptr;
  CQ_REQUIRE(a.info && a.logdet && a.trace, COQUI_B200_EINVAL, "dyson_run: result arrays missing");

  if (a.want_e) {
    logdet->assign(nw * nq, 0.0);
    trace->assign(nw * nq, make_double2(0, 0));
  }
  for (int64_t p0 = 0; p0 < nprob; p0 += nbq) {
    const int64_t nb = std::min(nbq, nprob - p0);
    const int64_t q0 = p0 % nq;
    unsigned char* Pi = a.PW + (size_t)p0 * NN * es;
    unsigned char* Mb = mpi ? Pi : Mb0;
    const float2* Lc = a.Lc;  // mixed form: complex64 factors, addressed periodically in q
    const float2* LHc = a.LHc;
    // M = L^H (Pi L)
    {
      Prof::Scope sc(a.prof, "dyson_M_gemm");
      if (a.mixed) {
        // P1 = L^H Pi  (Pi Hermitian: B(k, n) = Pi[k][n] = conj(Pi[n][k]))
        // Only P1's tiles on and above the diagonal are needed: the lower triangle of M reads
        // Q = P1^H at (a, j) with a >= i >= j.  The others are written as zeros, which only
        // meet the zeros of L^H in the next product (Np^3 / 3 products instead of Np^3 / 2).
        TcStructure s1;
        s1.a_upper = true;  // L^H upper triangular
        s1.upper_zero = true;
        s1.a_mod = nq;
        s1.a_q0 = q0;
        tc_cgemm_nt(LHc, false, false, Np, NN, Pi, false, true, Np, NN, (float2*)T1, Np, NN, Np,
                    Np, Np, nb, s, s1);
        // M = L^H Q with Q = Pi L = P1^H (Pi Hermitian): B(k, n) = Q[k][n] = conj(P1[n][k]).
        // With L^H upper the lower triangle of M needs k >= i only (Np^3 / 6 products).
        TcStructure s2;
        s2.a_upper = true;     // L^H upper triangular
        s2.a_mod = nq;
        s2.a_q0 = q0;
        s2.lower_only = true;  // M Hermitian: the Cholesky reads the lower triangle
        tc_cgemm_nt(LHc, false, false, Np, NN, T1, false, true, Np, NN, (float2*)Mb, Np, NN, Np, Np,
                    Np, nb, s, s2);
      } else {
        // the same two triangular products in FP64 (zgemm.cu): P1 = L^H Pi, M = L^H P1^H
        ZgemmArgs z1;
        z1.M = z1.N = z1.K = Np;
        z1.A = a.LH;
        z1.lda = Np;
        z1.sA = NN;
        z1.a_upper = true;
        z1.upper_zero = true;  // as in the mixed form: P1's upper tiles are the ones M reads
        z1.a_mod = nq;
        z1.a_q0 = q0;
        z1.B = (const double2*)Pi;
        z1.ldb = Np;
        z1.sB = NN;
        z1.C = (double2*)T1;
        z1.ldc = Np;
        z1.sC = NN;
        z1.batch = nb;
        zgemm(z1, s);
        ZgemmArgs z2 = z1;
        z2.upper_zero = false;
        z2.opB = 'C';
        z2.B = (const double2*)T1;
        z2.C = (double2*)Mb;
        z2.lower_only = true;
        zgemm(z2, s);
      }
    }
    // I - M = C C^H (FP64): log-determinant, trace of M, and the inverse
    // above one kInvGroup the mixed form's off-group blocks of the inverse come from the
    // tensor cores; the FP64 form forms the whole inverse in the factorisation kernel
    const bool tc_inverse = a.mixed && a.want_w && Np > kInvGroup;
    {
      Prof::Scope sc(a.prof, "dyson_chol_inv");
      if (!a.mixed)
        launch_chol_inv_c128((const double2*)Mb, A, a.logdet + p0, a.trace + p0, a.info + p0, Np,
                             nb, s);
      else if (tc_inverse) {
        // whole waves of the one-CTA kernel, and a remainder of less than a wave spread over
        // many CTAs per problem when that finishes sooner (identical results either way)
        const int64_t wave = chol_wave_size();
        const int64_t full = nb >= wave ? nb / wave * wave : 0, rest = nb - full;
        const float2* M0 = (const float2*)Mb;
        if (full > 0)
          launch_chol_group_inv(M0, A, a.logdet + p0, a.trace + p0, a.info + p0, Np, full, s);
        if (rest > 0 && chol_prefer_tiled(std::vector<int64_t>((size_t)rest, Np)))
          launch_chol_tiled_strided(M0 + full * NN, A + full * NN, a.logdet + p0 + full,
                                    a.trace + p0 + full, a.info + p0 + full, Np, rest, s);
        else if (rest > 0)
          launch_chol_group_inv(M0 + full * NN, A + full * NN, a.logdet + p0 + full,
                                a.trace + p0 + full, a.info + p0 + full, Np, rest, s);
      }
      else
        launch_chol_inv((const float2*)Mb, A, a.want_w ? (float2*)Y : nullptr, a.logdet + p0,
                        a.trace + p0, a.info + p0, Np, nb, s);
    }
    if (!a.want_w) continue;
    // W = L E L^H with E = (I - M)^{-1} - I = D + D^H + D^H D, D = C^{-1} - I: no
    // cancellation against V, so the split-TF32 products keep W to ~1e-8.
    if (a.mixed) {
      if (tc_inverse) {
        // U = C^{-H} by doubling: FP64 inverses of the kInvGroup diagonal groups, then for
        // each level b the pairs of diagonal blocks (r0: b, r1: b1) get
        //   U01 = -U00 C10^H U11
        // as two split-TF32 products.  Z holds U - I (the D^H of the W products), Zl holds
        // U^H - I where a later level needs it, Zc = -C off the groups.
        Prof::Scope sc(a.prof, "dyson_tc_inverse");
        float2* Z = (float2*)Y;
        float2* Zl = (float2*)Y + nbq * NN;
        float2* Zc = (float2*)T1;
        float2* S = (float2*)Mb;
        launch_chol_split(A, Z, Zl, Zc, Np, nb, s);
        for (int64_t b = kInvGroup; b < Np; b *= 2) {
          for (int64_t r0 = 0; r0 + b < Np; r0 += 2 * b) {
            const int64_t r1 = r0 + b, b1 = std::min(b, Np - r1);
            // S = U00 (-C10)^H  (b x b1, K = b): A = Z + I on the 00 block (upper)
            TcStructure t1;
            t1.a_upper = true;
            t1.a_ident = true;
            tc_cgemm_nt(Z + r0 * Np + r0, false, false, Np, NN, Zc + r1 * Np + r0, false, true,
                        Np, NN, S + r0 * Np + r1, Np, NN, b, b1, b, nb, s, t1);
            // U01 = S U11 with U11(k, n) = conj(Zl[n][k]) + delta  (b x b1, K = b1)
            TcStructure t2;
            t2.b_upper = true;
            t2.b_ident = true;
            tc_cgemm_nt(S + r0 * Np + r1, false, false, Np, NN, Zl + r1 * Np + r1, false, true,
                        Np, NN, Z + r0 * Np + r1, Np, NN, b, b1, b1, nb, s, t2);
            if (2 * b < Np) launch_block_adjoint(Z, Zl, Np, r0, r1, b, b1, nb, s);
          }
        }
      }
      const float2* Z = (const float2*)Y;  // DH = C^{-H} - I
      Prof::Scope sc(a.prof, "dyson_W_gemm");
      float2* F = (float2*)T1;
      float2* E = (float2*)Mb;
      // F = D^H D  (B(k, n) = D[k][n] = conj(DH[n][k]))
      TcStructure s3;
      s3.a_upper = true;     // D^H upper
      s3.b_lower = true;     // D lower
      s3.lower_only = true;  // F Hermitian
      tc_cgemm_nt(Z, false, false, Np, NN, Z, false, true, Np, NN, F, Np, NN, Np, Np, Np, nb, s, s3);
      const int64_t nt32 = (Np + 31) / 32;
      k_herm_sum<<<dim3((unsigned)(nt32 * (nt32 + 1) / 2), (unsigned)nb), 256, 0, s>>>(Z, F, E, Np);
      count_launch();
      // W is Hermitian: its lower triangle W_ij (j <= i) = sum_{k <= j} T_ik conj(L_jk) needs
      // T = L E only on and below the diagonal tiles, and the upper triangle is its mirror.
      // T = L E  (E Hermitian: B(k, n) = conj(E[n][k]))
      TcStructure s4;
      s4.a_lower = true;  // L lower
      s4.lower_only = true;
      s4.a_mod = nq;
      s4.a_q0 = q0;
      tc_cgemm_nt(Lc, false, false, Np, NN, E, false, true, Np, NN, F, Np, NN, Np, Np, Np, nb, s, s4);
      // W = T L^H  (B(k, n) = conj(L[n][k])), written over Pi
      TcStructure s5;
      s5.b_upper = true;  // B(k, n) = conj(L[n][k]) vanishes for k > n
      s5.lower_only = true;
      s5.b_mod = nq;
      s5.b_q0 = q0;
      tc_cgemm_nt(F, false, false, Np, NN, Lc, false, true, Np, NN, (float2*)Pi, Np, NN, Np, Np,
                  Np, nb, s, s5);
      launch_mirror_upper((float2*)Pi, Np, nb, s);
    } else {
      // the same W = L E L^H in FP64: Z = D^H, F = D^H D, E = Z + Z^H + F, T = L E, W = T L^H
      Prof::Scope sc(a.prof, "dyson_W_gemm");
      double2* Z = (double2*)T1;
      double2* F = (double2*)Mb;
      double2* E = A;  // the factorisation is not needed once Z holds C^{-H} - I
      launch_upper_minus_eye(A, Z, Np, nb, s);
      ZgemmArgs f;  // F = Z Z^H: Z upper, B(k, n) = conj(Z[n][k]) lower
      f.M = f.N = f.K = Np;
      f.opB = 'C';
      f.A = f.B = Z;
      f.lda = f.ldb = f.ldc = Np;
      f.sA = f.sB = f.sC = NN;
      f.C = F;
      f.batch = nb;
      f.a_upper = f.b_lower = f.lower_only = true;
      zgemm(f, s);
      const int64_t total = NN * nb;
      k_herm_sum_c128<<<grid_for(total, 256), 256, 0, s>>>(Z, F, E, Np, total);
      count_launch();
      CQ_CHECK_CUDA(cudaGetLastError());
      ZgemmArgs t;  // T = L E (lower tiles), L lower, E Hermitian (stored whole)
      t.M = t.N = t.K = Np;
      t.A = a.L;
      t.lda = t.ldb = t.ldc = Np;
      t.sA = t.sB = t.sC = NN;
      t.a_mod = nq;
      t.a_q0 = q0;
      t.a_lower = t.lower_only = true;
      t.B = E;
      t.C = F;
      t.batch = nb;
      zgemm(t, s);
      ZgemmArgs w;  // W = T L^H (lower tiles), B(k, n) = conj(L[n][k]) upper
      w.M = w.N = w.K = Np;
      w.opB = 'C';
      w.A = F;
      w.B = a.L;
      w.lda = w.ldb = w.ldc = Np;
      w.sA = w.sB = w.sC = NN;
      w.b_mod = nq;
      w.b_q0 = q0;
      w.b_upper = w.lower_only = true;
      w.C = (double2*)Pi;
      w.batch = nb;
      zgemm(w, s);
      mirror_upper<double2>((double2*)Pi, Np, nb, s, 0);
    }
  }
  if (!a.defer_check) {
    std::vector<int> info(nprob);
    CQ_CHECK_CUDA(cudaMemcpyAsync(info.data(), a.info, nprob * sizeof(int), cudaMemcpyDeviceToHost, s));
    if (a.want_e) {
      CQ_CHECK_CUDA(cudaMemcpyAsync(logdet->data(), a.logdet, nprob * sizeof(double),
                                    cudaMemcpyDeviceToHost, s));
      CQ_CHECK_CUDA(cudaMemcpyAsync(trace->data(), a.trace, nprob * sizeof(double2),
                                    cudaMemcpyDeviceToHost, s));
    }
    CQ_CHECK_CUDA(cudaStreamSynchronize(s));
    for (int64_t i = 0; i < nprob; ++i)
      if (info[i] != 0)
        throw Error(COQUI_B200_ENOTHPD, "I - L^H Pi L is not positive definite at (w=" +
                                            std::to_string(i / nq) + ", q=" + std::to_string(i % nq) +
                                            ")");
  }
}

}  // namespace cq
