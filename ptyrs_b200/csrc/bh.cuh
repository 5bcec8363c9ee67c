// pty-chi's bilinear Hessian of the amplitude cost on the device (physwkim/ptyrs
// engine/bh.rs:500-575), one frame per thread-block cluster: with the exit waves' first-order
// changes L_u = U·J u and L_v = U·J v along the displacements u = (u_O, u_P) and
// v = (v_O, v_P), J u = (u_P·O + P·u_O)·q, and the second-order one J″(u, v) =
// (u_P·v_O + v_P·u_O)·q, a frame's share of H(u, v) is
//   Re⟨g, J″(u, v)⟩ + 2·Σ_unmasked [(1 − d/a)·Σ_m Re(conj(L_u)·L_v) + d·c_u·c_v / a³]
// with g = Uᴴ(2·td) the gradient pass's exit-plane field (the term 2·Re⟨td, U·J″⟩ taken by
// Parseval in the exit plane, no transform), c_u = Σ_m Re(conj(U psi)·L_u) against the
// detector field the gradient pass kept, a = √Σ_m |U psi|² + 1e-8 and d = √I.
// Under the position model (engine/bh.rs:92-275, Patch sampling) each frame reads its moved
// planes M(P), M(u_P), M(v_P) in place of P, u_P, v_P; with refined offsets the displacements'
// offsets parts u_d, v_d add dW_u = M(u_P) + Σ_a u_da·∂_a M(P) in place of M(u_P) and to J″
// the term (Σ_a v_da·∂_a M(u_P) + u_da·∂_a M(v_P) + Σ_ab u_da·v_db·∂_a∂_b M(P))·O·q.
#pragma once
#include "frame.cuh"

namespace ptyb {

struct BhArgs {
  const float2* object;   // [nobj][nyo][nxo]
  const float2* probe;    // [nprobe][N][N]
  const float2* u_obj;    // u_O, laid out as the object
  const float2* u_probe;  // u_P, laid out as the probe
  const float2* v_obj;
  const float2* v_probe;
  const float2* quad;
  const float2* tw;
  const float* iobs;
  const int* frames;
  const int2* corners;
  double* out;            // [slot]: the frame's share of H(u, v)
  int nyo, nxo, nprobe, nobj;
  int same;               // v is u: one tangent transform per mode
  // U psi of every slot and mode as the gradient pass kept it, [slot][K][kx][ky] (the frame
  // kernel's unnormalised transform), and its exit-plane field g = Uᴴ(2·td), [slot][K][N][N].
  const float2* psi;
  const float2* g;
  // Position model (null without): every slot's moved planes [slot][K][N][N], M(P), M(u_P),
  // M(v_P); with refined offsets their offset derivatives (∂y, ∂x of each; ∂y∂y, ∂y∂x, ∂x∂x of
  // M(P)) and the displacements' offsets parts [slot][2] (dy, dx).
  const float2 *w, *tu, *tv;
  const float2 *dwy, *dwx, *dtuy, *dtux, *dtvy, *dtvx, *dwyy, *dwyx, *dwxx;
  const double *ud, *vd;
};

template <int N, int C>
__host__ __device__ constexpr size_t bh_smem_bytes() {
  using F = FrameShape<N, C>;
  return 2 * (size_t)F::H * F::L * sizeof(float2) + 4 * (size_t)F::H * (N + 1) * sizeof(float) +
         N * sizeof(float2) + 160 * sizeof(double);
}

template <int N, int C>
__global__ void __launch_bounds__(FrameShape<N, C>::T, 1) bh_hessian_kernel(BhArgs a) {
  using F = FrameShape<N, C>;
  constexpr int H = F::H, T = F::T, L = F::L, AS = N + 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* S1 = reinterpret_cast<float2*>(smem_raw);           // L_u, then L_v
  float* acc = reinterpret_cast<float*>(S1 + 2 * (size_t)H * L);  // [4][H][N + 1]
  double* red = reinterpret_cast<double*>(acc + 4 * H * AS + 2 * N);
  cg::cluster_group cluster = cg::this_cluster();
  const int r = C > 1 ? (int)cluster.block_rank() : 0;
  const int slot = blockIdx.x / C;
  const int f = a.frames[slot];
  const int2 corner = a.corners[f];
  const int tid = threadIdx.x;
  const int K = a.nprobe * a.nobj;
  // L_v's lines follow L_u's: line H + l of S1, swizzled as that line (transpose and the line
  // FFTs address both planes from S1)
  const int planes = a.same ? 1 : 2;
  constexpr float inv_n2 = 1.0f / ((float)N * (float)N);
  LineTwiddles<N> ltw;
  ltw.load(a.tw, tid % F::G);
  for (int i = tid; i < 4 * H * AS; i += T) acc[i] = 0.f;

  const bool moved = a.w != nullptr, pos = a.dwy != nullptr;
  float uy = 0.f, ux = 0.f, vy = 0.f, vx = 0.f;
  if (pos) {
    uy = (float)a.ud[2 * slot];
    ux = (float)a.ud[2 * slot + 1];
    vy = (float)a.vd[2 * slot];
    vx = (float)a.vd[2 * slot + 1];
  }
  double gterm = 0.0;
  for (int m = 0; m < K; ++m) {
    const int pm = m % a.nprobe, om = m / a.nprobe;
    const float2* po_m = a.psi + ((size_t)slot * K + m) * N * N + (size_t)r * H * N;
    const float2* g_m = a.g + ((size_t)slot * K + m) * N * N;
    // Exit-plane rows (shifted, as the frame kernel's) of J u and J v; J″(u, v) against g.
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int yl = idx / N, jx = idx % N;
      const int ny = (r * H + yl + N / 2) % N, nx = (jx + N / 2) % N;
      const size_t pi = ((size_t)pm * N + ny) * N + nx;
      const size_t si = ((size_t)slot * K + m) * N * N + (size_t)ny * N + nx;
      const size_t oi = ((size_t)om * a.nyo + corner.x + ny) * a.nxo + corner.y + nx;
      const float2 o = a.object[oi], q = a.quad[ny * N + nx];
      const float2 p = moved ? a.w[si] : a.probe[pi];
      float2 up = moved ? a.tu[si] : a.u_probe[pi];
      float2 vp = a.same ? up : moved ? a.tv[si] : a.v_probe[pi];
      const float2 uo = a.u_obj[oi];
      const float2 vo = a.same ? uo : a.v_obj[oi];
      float2 second = make_float2(0.f, 0.f);  // J″'s offsets terms, before ·O·q
      if (pos) {
        const float2 wy = a.dwy[si], wx = a.dwx[si];
        const float2 sy = a.dtuy[si], sx = a.dtux[si];
        const float2 ty = a.same ? sy : a.dtvy[si], tx = a.same ? sx : a.dtvx[si];
        second = cadd(cadd(cscale(sy, vy), cscale(sx, vx)), cadd(cscale(ty, uy), cscale(tx, ux)));
        second = cadd(second, cadd(cscale(a.dwyy[si], uy * vy),
                                   cadd(cscale(a.dwyx[si], uy * vx + ux * vy),
                                        cscale(a.dwxx[si], ux * vx))));
        up = cadd(up, cadd(cscale(wy, uy), cscale(wx, ux)));
        vp = a.same ? up : cadd(vp, cadd(cscale(wy, vy), cscale(wx, vx)));
      }
      S1[yl * L + (jx ^ swz(yl))] = cmul(cadd(cmul(up, o), cmul(p, uo)), q);
      float2 xuv;
      if (a.same) {
        xuv = cscale(cmul(cmul(up, uo), q), 2.f);
      } else {
        const int l2 = H + yl;
        S1[l2 * L + (jx ^ swz(l2))] = cmul(cadd(cmul(vp, o), cmul(p, vo)), q);
        xuv = cmul(cadd(cmul(up, vo), cmul(vp, uo)), q);
      }
      if (pos) xuv = cadd(xuv, cmul(cmul(second, o), q));
      const float2 gv = g_m[(size_t)ny * N + nx];
      gterm += (double)gv.x * xuv.x + (double)gv.y * xuv.y;
    }
    __syncthreads();
    all_lines<N, C, -1>(S1, planes * H, ltw);
    transpose<N, C>(S1, planes, cluster);
    all_lines<N, C, -1>(S1, planes * H, ltw);
    // Columns kx = r·H + c, elements ky: Σ|U psi|², Re(conj(L_u)·L_v), c_u and c_v terms.
#pragma unroll 2
    for (int idx = tid; idx < H * N; idx += T) {
      const int c = idx / N, ky = idx % N;
      const float2 po = po_m[(size_t)c * N + ky];
      const float2 lu = S1[c * L + (ky ^ swz(c))];
      const float2 lv = a.same ? lu : S1[(H + c) * L + (ky ^ swz(H + c))];
      acc[c * AS + ky] += cnorm2(po) * inv_n2;
      acc[(H + c) * AS + ky] += (lu.x * lv.x + lu.y * lv.y) * inv_n2;
      acc[(2 * H + c) * AS + ky] += (po.x * lu.x + po.y * lu.y) * inv_n2;
      acc[(3 * H + c) * AS + ky] += (po.x * lv.x + po.y * lv.y) * inv_n2;
    }
    __syncthreads();
  }
  const float* iobs = a.iobs + (size_t)f * N * N;
  double v[4] = {gterm, 0.0, 0.0, 0.0};
  for (int idx = tid; idx < H * N; idx += T) {
    const int c = idx % H, ky = idx / H;
    const float yo = iobs[ky * N + r * H + c];
    if (yo < 0.f) continue;
    const double amp = sqrt((double)acc[c * AS + ky]) + 1e-8, d = sqrt((double)yo);
    const double uv = acc[(H + c) * AS + ky];
    const double cu = acc[(2 * H + c) * AS + ky], cv = acc[(3 * H + c) * AS + ky];
    v[0] += 2.0 * ((1.0 - d / amp) * uv + d * cu * cv / (amp * amp * amp));
  }
  block_sum<T>(v, 1, red);
  csync<C>(cluster);
  if (r == 0 && tid == 0) {
    double h = 0.0;
    for (int q = 0; q < C; ++q) h += (C > 1 ? cluster.map_shared_rank(red, q) : red)[0];
    a.out[slot] = h;
  }
  csync<C>(cluster);
}

}  // namespace ptyb
