// Data-movement and element-wise kernels of the U-Net warm start (sm_100a).  The convolutions
// themselves are implicit GEMMs on the tcgen05 GEMM (gemm_tc.cu) over the im2col matrices built
// here.  Activations are NHWC; convolution K index = tap * C + c with tap = (dy+1)*3 + (dx+1),
// zero-padded to a multiple of 64.
#include <cuda_bf16.h>

#include "common.cuh"

namespace mw {

typedef __nv_bfloat16 bf16;

// X [B,H,W,C] (bf16) -> col [M = B*H*W, Kp] (bf16), 'same' 3x3 patches, zeros outside
__global__ void k_im2col(int B, int H, int W, int C, int Kp, const bf16* __restrict__ X, bf16* __restrict__ col) {
  const int64_t M = (int64_t)B * H * W;
  const int64_t total = M * Kp;
  const bf16 z = __float2bfloat16(0.f);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / Kp;
    const int k = (int)(i - p * Kp);
    bf16 v = z;
    if (k < 9 * C) {
      const int tap = k / C, c = k - tap * C;
      const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((int64_t)W * H));
      const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
      if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = X[(((int64_t)b * H + yy) * W + xx) * C + c];
    }
    col[i] = v;
  }
}

// transposed im2col: colT [Kp, ldT] (ldT >= M; columns p >= M are zero so the pixel dimension can
// be padded to the GEMM's K granularity)
__global__ void k_im2col_T(int B, int H, int W, int C, int Kp, int64_t ldT, const bf16* __restrict__ X,
                           bf16* __restrict__ colT) {
  const int64_t M = (int64_t)B * H * W;
  const int64_t total = ldT * Kp;
  const bf16 z = __float2bfloat16(0.f);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i / ldT);
    const int64_t p = i - (int64_t)k * ldT;
    bf16 v = z;
    if (k < 9 * C && p < M) {
      const int tap = k / C, c = k - tap * C;
      const int x = (int)(p % W), y = (int)((p / W) % H), b = (int)(p / ((int64_t)W * H));
      const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
      if (yy >= 0 && yy < H && xx >= 0 && xx < W) v = X[(((int64_t)b * H + yy) * W + xx) * C + c];
    }
    colT[i] = v;
  }
}

// fp32 master weights W [Cout, Kp_in] -> bf16 copy
__global__ void k_cast_bf16(int64_t n, const float* __restrict__ a, bf16* __restrict__ b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = __float2bfloat16(a[i]);
}

// Weights of the data-gradient convolution: Wt[ci][tap'*Cout + co] = W[co][(8-tap')*Cin + ci]
__global__ void k_w_bwd(int Cout, int Cin, int Kp_in, int Kp_out, const float* __restrict__ W, bf16* __restrict__ Wt) {
  const int64_t total = (int64_t)Cin * Kp_out;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int ci = (int)(i / Kp_out), k = (int)(i % Kp_out);
    float v = 0.f;
    if (k < 9 * Cout) {
      const int tp = k / Cout, co = k - tp * Cout;
      v = W[(int64_t)co * Kp_in + (8 - tp) * Cin + ci];
    }
    Wt[i] = __float2bfloat16(v);
  }
}

// dZ = dA * (A > 0 or !relu): bf16 [M, C], bf16 transposed [C, ldT] (columns >= M untouched), fp32 [M, C]
__global__ void k_relu_grad(int64_t M, int C, int relu, int64_t ldT, const float* __restrict__ dA,
                            const bf16* __restrict__ A, bf16* __restrict__ dZ, bf16* __restrict__ dZT,
                            float* __restrict__ dZ32) {
  const int64_t total = M * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / C;
    const int c = (int)(i - p * C);
    float g = dA[i];
    if (relu && !(__bfloat162float(A[i]) > 0.f)) g = 0.f;
    const bf16 gb = __float2bfloat16(g);
    dZ[i] = gb;
    dZT[(int64_t)c * ldT + p] = gb;
    dZ32[i] = g;
  }
}

// column sums of X [M, C] (fp32): one block per column, deterministic
__global__ void k_colsum(int64_t M, int C, const float* __restrict__ X, float* __restrict__ out) {
  __shared__ double sh[32];
  const int c = blockIdx.x;
  double s = 0;
  for (int64_t p = threadIdx.x; p < M; p += blockDim.x) s += X[p * C + c];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    out[c] = (float)t;
  }
}

// 2x2 average pooling, NHWC bf16
__global__ void k_avgpool2(int B, int H, int W, int C, const bf16* __restrict__ X, bf16* __restrict__ Y) {
  const int h = H / 2, w = W / 2;
  const int64_t total = (int64_t)B * h * w * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int x = (int)(q % w), y = (int)((q / w) % h), b = (int)(q / ((int64_t)w * h));
    const bf16* s = X + (((int64_t)b * H + 2 * y) * W + 2 * x) * C + c;
    float v = __bfloat162float(s[0]) + __bfloat162float(s[C]) + __bfloat162float(s[(int64_t)W * C]) +
              __bfloat162float(s[(int64_t)W * C + C]);
    Y[i] = __float2bfloat16(0.25f * v);
  }
}

// gradient of avg pooling: dX[b,y,x,c] (+)= dY[b,y/2,x/2,c] / 4   (fp32)
__global__ void k_avgpool2_bwd(int B, int H, int W, int C, const float* __restrict__ dY, float* __restrict__ dX,
                               int accumulate) {
  const int64_t total = (int64_t)B * H * W * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int x = (int)(q % W), y = (int)((q / W) % H), b = (int)(q / ((int64_t)W * H));
    const float g = 0.25f * dY[(((int64_t)b * (H / 2) + y / 2) * (W / 2) + x / 2) * C + c];
    dX[i] = accumulate ? dX[i] + g : g;
  }
}

// nearest 2x upsampling of X [B,h,w,C] into channels [c0, c0+C) of Y [B,2h,2w,Ctot]
__global__ void k_upsample2_into(int B, int h, int w, int C, int Ctot, int c0, const bf16* __restrict__ X,
                                 bf16* __restrict__ Y) {
  const int H = 2 * h, W = 2 * w;
  const int64_t total = (int64_t)B * H * W * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int x = (int)(q % W), y = (int)((q / W) % H), b = (int)(q / ((int64_t)W * H));
    Y[q * Ctot + c0 + c] = X[(((int64_t)b * h + y / 2) * w + x / 2) * C + c];
  }
}

// copy X [.., C] into channels [c0, c0+C) of Y [.., Ctot]
__global__ void k_copy_channels(int64_t P, int C, int Ctot, int c0, const bf16* __restrict__ X, bf16* __restrict__ Y) {
  const int64_t total = P * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / C;
    const int c = (int)(i - p * C);
    Y[p * Ctot + c0 + c] = X[i];
  }
}

// gradient of the upsample into a concat: dX[b,y,x,c] = sum of the 4 fine cells' dY[.., c0+c]
__global__ void k_upsample2_bwd(int B, int h, int w, int C, int Ctot, int c0, const float* __restrict__ dY,
                                float* __restrict__ dX) {
  const int W = 2 * w;
  const int64_t total = (int64_t)B * h * w * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const int64_t q = i / C;
    const int x = (int)(q % w), y = (int)((q / w) % h), b = (int)(q / ((int64_t)w * h));
    const int64_t r0 = ((int64_t)b * 2 * h + 2 * y) * W + 2 * x;
    float s = dY[r0 * Ctot + c0 + c] + dY[(r0 + 1) * Ctot + c0 + c] + dY[(r0 + W) * Ctot + c0 + c] +
              dY[(r0 + W + 1) * Ctot + c0 + c];
    dX[i] = s;
  }
}

// dX[.., c] (+)= dY[.., c0 + c]   (channel slice of a concat gradient)
__global__ void k_slice_grad(int64_t P, int C, int Ctot, int c0, const float* __restrict__ dY, float* __restrict__ dX,
                             int accumulate) {
  const int64_t total = P * C;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t p = i / C;
    const int c = (int)(i - p * C);
    const float g = dY[p * Ctot + c0 + c];
    dX[i] = accumulate ? dX[i] + g : g;
  }
}

// MSE: loss = mean((y - t)^2); dy = 2 (y - t) / n ; partial sums of the loss per block
__global__ void k_mse(int64_t n, const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy,
                      double* __restrict__ loss_part) {
  __shared__ double sh[32];
  double s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    dy[i] = 2.f * d / (float)n;
    s += (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t2 = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t2 += sh[w];
    loss_part[blockIdx.x] = t2;
  }
}

// Adam (decoupled weight decay off): fp32 master weights, moments, gradient; bf16 copy refreshed
__global__ void k_adam(int64_t n, float* __restrict__ w, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, float lr, float b1, float b2, float eps, float bc1, float bc2,
                       bf16* __restrict__ w16) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16(wi);
  }
}

// ---- between finite-element fields and the element-centre grid of the network ----
// mean of log10(eta_e) -> stats[0]; velocity scale Ra / 10^mean -> stats[1]  (one block)
__global__ void k_feature_stats(int64_t nel, const double* __restrict__ eta_e, double Ra, double* __restrict__ stats) {
  __shared__ double sh[32];
  double s = 0;
  for (int64_t e = threadIdx.x; e < nel; e += blockDim.x) s += log10(eta_e[e]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    const double m = t / (double)nel;
    stats[0] = m;
    stats[1] = Ra / pow(10.0, m);
  }
}

// features [gzp, gxp, 2] bf16 on the network grid (f x f elements per cell, averaged):
// T at the element centre nodes, (log10 eta_e - mean) / 2.5.  The grid of the mesh is nelz/f x
// nelx/f; a network grid gzp x gxp larger than that (the network needs multiples of 8) repeats the
// last row and column (replicate padding).
__global__ void k_features(mw_box b, int f, int gxp, int gzp, const double* __restrict__ T,
                           const double* __restrict__ eta_e, const double* __restrict__ stats, bf16* __restrict__ X) {
  const int gx = b.nelx / f, gz = b.nelz / f;
  const int64_t ncell = (int64_t)gxp * gzp;
  const int nnx = 2 * b.nelx + 1;
  const double inv = 1.0 / ((double)f * f);
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncell; c += (int64_t)gridDim.x * blockDim.x) {
    const int cx = min((int)(c % gxp), gx - 1), cz = min((int)(c / gxp), gz - 1);
    double st = 0, se = 0;
    for (int a = 0; a < f; ++a)
      for (int d = 0; d < f; ++d) {
        const int ex = cx * f + d, ez = cz * f + a;
        st += T ? T[q2_node(ex, ez, 8, nnx)] : 0.0;
        se += log10(eta_e[(int64_t)ez * b.nelx + ex]);
      }
    X[2 * c] = __float2bfloat16((float)(st * inv));
    X[2 * c + 1] = __float2bfloat16((float)((se * inv - stats[0]) / 2.5));
  }
}

// hydrostatic pressure of the reference density: ghyd * (Lz/2 - z) (zero mean over a uniform lattice)
__device__ __forceinline__ double p_hydro(const mw_box& b, double ghyd, double z) { return ghyd * (0.5 * b.Lz - z); }

// Output channels of the network (NC = 5): 0, 1 = u, w / sv; 2 = (p - hydrostatic) / sp; 3, 4 =
// log10 sv, log10 sp, constant maps whose mean over the grid is the prediction of the two scales.
// sv, sp are the RMS of the velocity (units stats[1]) and of the dynamic pressure (units pscale)
// over the element centres, so every channel the loss sees is O(1) whatever Ra and the contrast.
constexpr int NC = 5;

// element-centre values of a solution in network units before normalisation
__device__ __forceinline__ void centre_values(const mw_box& b, const double* solV, const double* solP, double vs,
                                              double pscale, double ghyd, int64_t e, double* u, double* w, double* p) {
  const int nnx = 2 * b.nelx + 1;
  const int ex = (int)(e % b.nelx), ez = (int)(e / b.nelx);
  const int64_t c = q2_node(ex, ez, 8, nnx);
  *u = solV[2 * c] / vs;
  *w = solV[2 * c + 1] / vs;
  double pp = 0;
  for (int k = 0; k < 4; ++k) pp += solP[q1_node(ex, ez, k, b.nelx)];
  *p = (0.25 * pp - p_hydro(b, ghyd, (ez + 0.5) * b.hz)) / pscale;
}

// scales[0] = sv = sqrt(mean (u^2 + w^2) / 2), scales[1] = sp = sqrt(mean p^2) (one block)
__global__ void k_target_scales(mw_box b, const double* __restrict__ solV, const double* __restrict__ solP,
                                const double* __restrict__ stats, double pscale, double ghyd,
                                double* __restrict__ scales) {
  __shared__ double sh[32];
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  double a = 0, c = 0;
  for (int64_t e = threadIdx.x; e < nel; e += blockDim.x) {
    double u, w, p;
    centre_values(b, solV, solP, stats[1], pscale, ghyd, e, &u, &w, &p);
    a += 0.5 * (u * u + w * w);
    c += p * p;
  }
  for (int o = 16; o > 0; o >>= 1) { a += __shfl_down_sync(0xffffffffu, a, o); c += __shfl_down_sync(0xffffffffu, c, o); }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) sh[wid] = a;
  __syncthreads();
  double ta = 0;
  if (threadIdx.x == 0) for (int i = 0; i < nw; ++i) ta += sh[i];
  __syncthreads();
  if (lane == 0) sh[wid] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tc = 0;
    for (int i = 0; i < nw; ++i) tc += sh[i];
    scales[0] = fmax(sqrt(ta / (double)nel), 1e-300);
    scales[1] = fmax(sqrt(tc / (double)nel), 1e-300);
  }
}

// training targets [nelz, nelx, NC] fp32 from a solution and its scales
__global__ void k_targets(mw_box b, const double* __restrict__ solV, const double* __restrict__ solP,
                          const double* __restrict__ stats, double pscale, double ghyd,
                          const double* __restrict__ scales, float* __restrict__ Y) {
  const int64_t nel = (int64_t)b.nelx * b.nelz;
  const double sv = scales[0], spp = scales[1];
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nel; e += (int64_t)gridDim.x * blockDim.x) {
    double u, w, p;
    centre_values(b, solV, solP, stats[1], pscale, ghyd, e, &u, &w, &p);
    float* y = Y + NC * e;
    y[0] = (float)(u / sv);
    y[1] = (float)(w / sv);
    y[2] = (float)(p / spp);
    y[3] = (float)log10(sv);
    y[4] = (float)log10(spp);
  }
}

// predicted scales from channels 3, 4: scales = 10^mean over the mesh's cells gx x gz of the
// network grid (row length gxp) (one block)
__global__ void k_pred_scales(int gx, int gz, int gxp, const float* __restrict__ Y, double* __restrict__ scales) {
  __shared__ double sh[64];
  double a = 0, c = 0;
  const int64_t ncell = (int64_t)gx * gz;
  for (int64_t k = threadIdx.x; k < ncell; k += blockDim.x) {
    const int64_t i = (k / gx) * gxp + k % gx;
    a += Y[NC * i + 3];
    c += Y[NC * i + 4];
  }
  for (int o = 16; o > 0; o >>= 1) { a += __shfl_down_sync(0xffffffffu, a, o); c += __shfl_down_sync(0xffffffffu, c, o); }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (lane == 0) { sh[wid] = a; sh[32 + wid] = c; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0, tc = 0;
    for (int i = 0; i < nw; ++i) { ta += sh[i]; tc += sh[32 + i]; }
    scales[0] = pow(10.0, ta / (double)ncell);
    scales[1] = pow(10.0, tc / (double)ncell);
  }
}

// prediction [nelz/f, nelx/f, NC] -> Stokes initial guess: solV (interleaved u, w on the Q2
// lattice, bilinear between network-cell centres, fixed dofs 0) and solP (Q1 nodes, bilinear
// dynamic pressure + hydrostatic pressure); scales = (sv, sp)
__global__ void k_to_fields(mw_box b, int f, int gxp, const float* __restrict__ Y, const double* __restrict__ stats,
                            double pscale, double ghyd, const double* __restrict__ scales,
                            const uint8_t* __restrict__ fix, double* __restrict__ solV, double* __restrict__ solP) {
  const int nnx = 2 * b.nelx + 1, nnz = 2 * b.nelz + 1;
  const int gxn = b.nelx / f, gzn = b.nelz / f;          // the mesh's cells of the network grid (rows gxp long)
  const int64_t nn = (int64_t)nnx * nnz;
  const int64_t np = (int64_t)(b.nelx + 1) * (b.nelz + 1);
  const double vs = stats[1] * scales[0], ps = pscale * scales[1];
  auto at = [&](int cx, int cz, int ch) -> double {
    cx = cx < 0 ? 0 : (cx >= gxn ? gxn - 1 : cx);
    cz = cz < 0 ? 0 : (cz >= gzn ? gzn - 1 : cz);
    return (double)Y[((int64_t)cz * gxp + cx) * NC + ch];
  };
  auto bilin = [&](double gx, double gz, int ch) -> double {
    const int x0 = (int)floor(gx), z0 = (int)floor(gz);
    const double fx = gx - x0, fz = gz - z0;
    return (1 - fz) * ((1 - fx) * at(x0, z0, ch) + fx * at(x0 + 1, z0, ch)) +
           fz * ((1 - fx) * at(x0, z0 + 1, ch) + fx * at(x0 + 1, z0 + 1, ch));
  };
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn + np; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < nn) {
      const int ix = (int)(i % nnx), iz = (int)(i / nnx);
      const double gx = ix / (2.0 * f) - 0.5, gz = iz / (2.0 * f) - 0.5;   // network-cell-centre coordinates
      for (int c = 0; c < 2; ++c) solV[2 * i + c] = fix[2 * i + c] ? 0.0 : bilin(gx, gz, c) * vs;
    } else {
      const int64_t n = i - nn;
      const int px = (int)(n % (b.nelx + 1)), pz = (int)(n / (b.nelx + 1));
      solP[n] = bilin(px / (double)f - 0.5, pz / (double)f - 0.5, 2) * ps + p_hydro(b, ghyd, pz * b.hz);
    }
  }
}

}  // namespace mw

using namespace mw;

extern "C" {

#define MW_GRID(n) grid_for((n), 256), 256, 0, (cudaStream_t)stream

int mw_unet_im2col(int32_t B, int32_t H, int32_t W, int32_t C, int32_t Kp, int32_t transposed, int64_t ldT,
                   const void* X, void* col, void* stream) {
  if (Kp < 9 * C || (Kp % 64) != 0) return MW_ERR_BAD_ARG;
  const int64_t M = (int64_t)B * H * W;
  if (transposed) {
    if (ldT < M) return MW_ERR_BAD_ARG;
    k_im2col_T<<<MW_GRID(ldT * Kp)>>>(B, H, W, C, Kp, ldT, (const bf16*)X, (bf16*)col);
  } else {
    k_im2col<<<MW_GRID(M * Kp)>>>(B, H, W, C, Kp, (const bf16*)X, (bf16*)col);
  }
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_cast_bf16(int64_t n, const float* a, void* b, void* stream) {
  k_cast_bf16<<<MW_GRID(n)>>>(n, a, (bf16*)b);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_weights_bwd(int32_t Cout, int32_t Cin, int32_t Kp_in, int32_t Kp_out, const float* W, void* Wt,
                        void* stream) {
  if (Kp_out < 9 * Cout || Kp_in < 9 * Cin) return MW_ERR_BAD_ARG;
  k_w_bwd<<<MW_GRID((int64_t)Cin * Kp_out)>>>(Cout, Cin, Kp_in, Kp_out, W, (bf16*)Wt);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_relu_grad(int64_t M, int32_t C, int32_t relu, int64_t ldT, const float* dA, const void* A, void* dZ,
                      void* dZT, float* dZ32, void* stream) {
  if (ldT < M) return MW_ERR_BAD_ARG;
  k_relu_grad<<<MW_GRID(M * C)>>>(M, C, relu, ldT, dA, (const bf16*)A, (bf16*)dZ, (bf16*)dZT, dZ32);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_colsum(int64_t M, int32_t C, const float* X, float* out, void* stream) {
  k_colsum<<<C, 256, 0, (cudaStream_t)stream>>>(M, C, X, out);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_avgpool2(int32_t B, int32_t H, int32_t W, int32_t C, const void* X, void* Y, void* stream) {
  k_avgpool2<<<MW_GRID((int64_t)B * (H / 2) * (W / 2) * C)>>>(B, H, W, C, (const bf16*)X, (bf16*)Y);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_avgpool2_bwd(int32_t B, int32_t H, int32_t W, int32_t C, const float* dY, float* dX, int32_t accumulate,
                         void* stream) {
  k_avgpool2_bwd<<<MW_GRID((int64_t)B * H * W * C)>>>(B, H, W, C, dY, dX, accumulate);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_upsample2_into(int32_t B, int32_t h, int32_t w, int32_t C, int32_t Ctot, int32_t c0, const void* X,
                           void* Y, void* stream) {
  k_upsample2_into<<<MW_GRID((int64_t)B * 4 * h * w * C)>>>(B, h, w, C, Ctot, c0, (const bf16*)X, (bf16*)Y);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_copy_channels(int64_t P, int32_t C, int32_t Ctot, int32_t c0, const void* X, void* Y, void* stream) {
  k_copy_channels<<<MW_GRID(P * C)>>>(P, C, Ctot, c0, (const bf16*)X, (bf16*)Y);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_upsample2_bwd(int32_t B, int32_t h, int32_t w, int32_t C, int32_t Ctot, int32_t c0, const float* dY,
                          float* dX, void* stream) {
  k_upsample2_bwd<<<MW_GRID((int64_t)B * h * w * C)>>>(B, h, w, C, Ctot, c0, dY, dX);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_slice_grad(int64_t P, int32_t C, int32_t Ctot, int32_t c0, const float* dY, float* dX, int32_t accumulate,
                       void* stream) {
  k_slice_grad<<<MW_GRID(P * C)>>>(P, C, Ctot, c0, dY, dX, accumulate);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_mse(int64_t n, const float* y, const float* t, float* dy, double* loss_part, int32_t nparts,
                void* stream) {
  if (nparts < 1) return MW_ERR_BAD_ARG;
  k_mse<<<nparts, 256, 0, (cudaStream_t)stream>>>(n, y, t, dy, loss_part);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_adam(int64_t n, float* w, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
                 float bc1, float bc2, void* w16, void* stream) {
  k_adam<<<MW_GRID(n)>>>(n, w, m, v, g, lr, b1, b2, eps, bc1, bc2, (bf16*)w16);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_features_padded(mw_box box, int32_t f, int32_t gxp, int32_t gzp, const double* T, const double* eta_e,
                            double Ra, double* stats, void* X, void* stream) {
  if (f < 1 || box.nelx % f || box.nelz % f || gxp < box.nelx / f || gzp < box.nelz / f) return MW_ERR_BAD_ARG;
  const int64_t nel = (int64_t)box.nelx * box.nelz;
  k_feature_stats<<<1, 1024, 0, (cudaStream_t)stream>>>(nel, eta_e, Ra, stats);
  MW_CHECK_LAUNCH();
  k_features<<<MW_GRID((int64_t)gxp * gzp)>>>(box, f, gxp, gzp, T, eta_e, stats, (bf16*)X);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_features(mw_box box, int32_t f, const double* T, const double* eta_e, double Ra, double* stats, void* X,
                     void* stream) {
  if (f < 1) return MW_ERR_BAD_ARG;
  return mw_unet_features_padded(box, f, box.nelx / f, box.nelz / f, T, eta_e, Ra, stats, X, stream);
}

int mw_unet_to_fields_padded(mw_box box, int32_t f, int32_t gxp, const float* Y, const double* stats, double pscale,
                             double ghyd, double* scales, const uint8_t* bc_fix_V, double* solV, double* solP,
                             void* stream) {
  if (f < 1 || box.nelx % f || box.nelz % f || !scales || gxp < box.nelx / f) return MW_ERR_BAD_ARG;
  k_pred_scales<<<1, 1024, 0, (cudaStream_t)stream>>>(box.nelx / f, box.nelz / f, gxp, Y, scales);
  MW_CHECK_LAUNCH();
  const int64_t n = (int64_t)(2 * box.nelx + 1) * (2 * box.nelz + 1) + (int64_t)(box.nelx + 1) * (box.nelz + 1);
  k_to_fields<<<MW_GRID(n)>>>(box, f, gxp, Y, stats, pscale, ghyd, scales, bc_fix_V, solV, solP);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

int mw_unet_to_fields(mw_box box, int32_t f, const float* Y, const double* stats, double pscale, double ghyd,
                      double* scales, const uint8_t* bc_fix_V, double* solV, double* solP, void* stream) {
  if (f < 1) return MW_ERR_BAD_ARG;
  return mw_unet_to_fields_padded(box, f, box.nelx / f, Y, stats, pscale, ghyd, scales, bc_fix_V, solV, solP, stream);
}

int mw_unet_targets(mw_box box, const double* solV, const double* solP, const double* stats, double pscale,
                    double ghyd, double* scales, float* Y, void* stream) {
  if (!scales) return MW_ERR_BAD_ARG;
  const int64_t nel = (int64_t)box.nelx * box.nelz;
  k_target_scales<<<1, 1024, 0, (cudaStream_t)stream>>>(box, solV, solP, stats, pscale, ghyd, scales);
  MW_CHECK_LAUNCH();
  k_targets<<<MW_GRID(nel)>>>(box, solV, solP, stats, pscale, ghyd, scales, Y);
  MW_CHECK_LAUNCH();
  return MW_OK;
}

}  // extern "C"
