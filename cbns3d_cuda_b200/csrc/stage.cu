// stage.cu - one SSP-RK3 stage in one kernel: inviscid WENO5-char/LF fluxes in
// all three directions, their differences, the viscous divergence (formed
// ahead of it by visc_div_kernel, visc.cu), division by J and the Shu-Osher
// stage combination, for every interior node.
//
// Replaces, for one stage, the reference's
//   calc_numerical_flux  (src/calc_numerical_flux.cu:15-74; three face kernels
//                         writing Ep/Fp/Gp to HBM)
//   update_rk3 / rk3_kernel     (src/time_integration.cu:15-40,
//                                src/runge_kutta_kernel.cu:13-80)
// and, in stage 3 of an inviscid step, the per-node half of calc_dt
// (src/time_step_kernel.cu:13-96) for interior nodes.
//
// Tiling (2.5D).  A CTA of 256 threads owns a TI x TJ = 16 x 15 column of
// interior nodes and marches it through a chunk of k planes.  Per plane:
//   ring   : the conservative state of the column on the 6 planes k-2..k+3
//            (stencil of the k-faces), loaded one new plane per step;
//   plane  : plane k with a 3-node halo in i and j (stencils of i/j faces);
//   areas  : the node area vectors J*grad(xi) on the i-face nodes and
//            J*grad(eta) on the j-face nodes of plane k (face normals);
//   round A: the 17 x 15 i-faces of plane k  (thread f -> face f, f < 255)
//   round B: the 16 x 16 j-faces of plane k  (thread f -> face f)
//   round C: the k+1/2 face of each column   (thread t -> column t, t < 240);
//            the k-1/2 flux and the column's J*grad(zeta) are carried in
//            registers from the previous plane.
// Every thread computes 3 faces per plane; face fluxes never leave the SM and
// no global load sits inside a face evaluation.
// Staging.  The FP32 kernels built for 2 or 3 CTAs per SM stage the next
// plane's halo (raw FP64 state) and face-node area vectors (FP32 copies) by
// TMA: one thread issues six 4-D box copies (tma.cuh) right after the current
// plane's staging barrier, completing on an mbarrier per plane parity, so they
// travel while the current plane's three flux rounds run; the ring column goes
// through registers (fetched a plane early, rounded to FP32 on the way into
// shared memory).  The FP64 kernel and the 4-CTA hybrid variant, which have no
// shared memory to spare for a second plane, stage synchronously.
// HBM traffic per node and stage: the stage input (40 B, halos from L2),
// area vectors and 1/J (80 B; the FP32 kernels stage FP32 copies of the xi
// and eta vectors, 56 B), the RK base (0-40 B) and the output (40 B).
//
// Hybrid (HYB): each face's sensor decision selects the linear upwind-5 flux,
// evaluated here, or the characteristic WENO5 flux, evaluated before this
// kernel by the WENO5-face pass (weno_faces.cu) and read from its face array.
// The decisions of plane k+1 are read while plane k is computed, and the
// WENO5 fluxes of plane k are asked into L1 before the plane's staging, so
// the face rounds wait on neither.  Holding no WENO5 code, the hybrid kernel
// runs at 3 CTAs per SM.
#include <type_traits>

#include "cbns_common.cuh"
#include "face_flux.cuh"
#include "stage.cuh"
#include "tma.cuh"

namespace cbns {

namespace {

constexpr int TI = 16, TJ = 15, H = 3;
constexpr int PW = TI + 2 * H;  // 22
constexpr int PH = TJ + 2 * H;  // 21
constexpr int NC = TI * TJ;     // 240 columns
constexpr int NT = 256;         // threads
constexpr int NFI = (TI + 1) * TJ;  // 255 i-faces
constexpr int NFJ = TI * (TJ + 1);  // 256 j-faces
// the face rounds' thread mapping (face_a, face_b in stage_body): one j-face
// per thread; i-faces on 7 warps of two 16-face rows and one of a row and the
// 15 faces of the last column
static_assert(NFJ == NT && TI == 16 && TJ == 15, "face mapping of the face rounds");
static_assert(NFI == 7 * 32 + 16 + TJ, "face mapping of the face rounds");
constexpr int NSX = (TI + 2) * TJ;  // i-face nodes (i0-1 .. i0+16)
constexpr int NSY = TI * (TJ + 2);  // j-face nodes (j0-1 .. j0+15)
constexpr int NHI = 2 * H * TJ, NHJ = 2 * H * TI;  // halo nodes of a plane: i-halo, j-halo

// Area vectors of the face nodes are staged in the flux precision: the flux
// converts them to it anyway (the FP32 kernels read FP32 copies made once with
// the metrics); the FP64 kernel keeps them exact.
template <typename R>
using AreaT = typename std::conditional<sizeof(R) == 4, float, double>::type;

__device__ __forceinline__ void prefetch_l1(const void* p) {
  asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}
__device__ __forceinline__ void prefetch_l2(const void* p) {
  asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// PWT: row pitch of the plane buffer (PW; 24 in the FP64 TMA kernel, whose
// plane is one TMA box starting at tile x = -4)
template <typename S, typename R, int PWT = PW>
struct Smem {
  S ring[6][NEQ][NC];
  S plane[NEQ][PH][PWT];
  R fi[NEQ][TJ][TI + 1];
  R fj[NEQ][TJ + 1][TI];
};

// Face-node area vectors of one plane, staged by the synchronous kernels.
template <typename R>
struct AreaSync {
  AreaT<R> sx[3][TJ][TI + 2];  // J*grad(xi) at node (i0-1+c, j0+r)
  AreaT<R> sy[3][TJ + 2][TI];  // J*grad(eta) at node (i0+c, j0-1+r)
};

// TMA staging of the FP32 kernels, each box as the copy writes it (x fastest,
// then rows, then fields): plane k+1's halo (raw FP64; one buffer, refilled
// after plane k's halo was converted) and the face-node area vectors of planes
// k and k+1 (two buffers).  Box x origins sit on 16-byte boundaries: the i-side
// halo boxes start at i0-4 and i0+16, the xi box at i0-4 (node i0-1+c at
// column c+3), the j-side and eta boxes at i0.
struct TmaSmem {
  alignas(128) double hl[NEQ][TJ][4];  // x = i0-4 .. i0-1, rows j0 .. j0+14
  alignas(128) double hr[NEQ][TJ][4];  // x = i0+16 .. i0+19
  alignas(128) double hb[NEQ][H][TI];  // x = i0 .. i0+15, rows j0-3 .. j0-1
  alignas(128) double ht[NEQ][H][TI];  // rows j0+15 .. j0+17
  struct Area {
    alignas(128) float xi[3][TJ][24];      // J*grad(xi), x = i0-4 .. i0+19, rows j0 .. j0+14
    alignas(128) float eta[3][TJ + 2][TI];  // J*grad(eta), x = i0 .. i0+15, rows j0-1 .. j0+15
  } area[2];
  alignas(8) unsigned long long bar[2];  // one per plane parity
};
// bytes of one plane's six boxes (the mbarrier's transaction count)
constexpr unsigned kTmaBytes =
    (unsigned)(sizeof(double) * NEQ * (2 * TJ * 4 + 2 * H * TI) + sizeof(float) * 3 * (TJ * 24 + (TJ + 2) * TI));

// TMA staging of the FP64 kernel: the ring column of a plane lands in its ring
// slot (box 16 x 15 x 1 x 5, the slot's [field][row][col] layout), the whole
// plane with its halo in the plane buffer (box 24 x 21 x 1 x 5 from tile x =
// -4, row pitch 24), the face-node area vectors (FP64) here; all single
// buffers, refilled for the next plane once the current plane's flux rounds
// are over, so the copies travel during the RK update.
struct TmaSmem64 {
  alignas(128) double xi[3][TJ][24];      // J*grad(xi), x = i0-4 .. i0+19, rows j0 .. j0+14
  alignas(128) double eta[3][TJ + 2][TI];  // J*grad(eta), x = i0 .. i0+15, rows j0-1 .. j0+15
  alignas(8) unsigned long long bar[2];
};
// bytes of the warm-up set (the ring's first six planes) and of a plane's set
// (its ring column three planes ahead, the plane with halo, the area vectors)
constexpr unsigned kTma64Warm = (unsigned)(6 * sizeof(double) * NEQ * NC);
constexpr unsigned kTma64Plane =
    (unsigned)(sizeof(double) * (NEQ * NC + NEQ * PH * 24 + 3 * TJ * 24 + 3 * (TJ + 2) * TI));

constexpr size_t round_to(size_t x, size_t m) { return (x + m - 1) / m * m; }

// dynamic shared memory: Smem, then (FP32 TMA kernels) TmaSmem on a 128-byte
// boundary found at run time, (the FP64 TMA kernel) Smem and TmaSmem64 from a
// 128-byte boundary, or (synchronous kernels) AreaSync
template <typename R, int NB, bool TMA>
__host__ __device__ constexpr size_t stage_smem() {
  return (TMA && sizeof(R) == 4)   ? round_to(sizeof(Smem<R, R>), 16) + 128 + sizeof(TmaSmem)
         : (TMA && sizeof(R) == 8) ? 128 + round_to(sizeof(Smem<R, R, 24>), 128) + sizeof(TmaSmem64)
                                   : round_to(sizeof(Smem<R, R>), 16) + sizeof(AreaSync<R>);
}

// NB = CTAs per SM the register budget is cut for: FP64 always 2 (shared
// memory allows no more); the split FP32 kernel is built for 2 (128
// registers) and 3 (80 registers, some spills), the hybrid for 2, 3 and 4 (64
// registers, no asynchronous staging); cbns_autotune keeps the fastest.
// HYB: hybrid flux (learned-sensor decision per face, see the flux lambda);
// it evaluates only the linear faces and holds no WENO5 code.
// The work of one CTA: tile `tile` of the block's (i, j) tiling, k chunk `kc`.
// TMA: TMA staging (FP32: halo and area vectors; FP64: ring column, plane and
// area vectors), else synchronous loads.
template <typename R, bool VISC, int MODE, int NB, bool HYB, bool TMA>
__device__ __forceinline__ void stage_body(const StageArgs& a, const StageMaps* tm, int tile, int kc,
                                           unsigned char* smem_raw) {
  using S = R;  // shared-memory storage type
  constexpr bool kTma = TMA && sizeof(R) == 4;
  constexpr bool kTma64 = TMA && sizeof(R) == 8;
  constexpr int PWT = kTma64 ? 24 : PW;  // plane row pitch
  constexpr int X0 = kTma64 ? 1 : 0;     // plane column of tile x = -H, minus H
  using SM = Smem<S, R, PWT>;
  unsigned char* base =
      kTma64 ? reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127))
             : smem_raw;
  SM& sm = *reinterpret_cast<SM*>(base);
  unsigned char* tail = base + round_to(sizeof(SM), kTma64 ? 128 : 16);
  TmaSmem* ts = reinterpret_cast<TmaSmem*>((reinterpret_cast<uintptr_t>(tail) + 127) & ~uintptr_t(127));
  TmaSmem64* t64 = reinterpret_cast<TmaSmem64*>(tail);
  AreaSync<R>* asy = reinterpret_cast<AreaSync<R>*>(tail);

  const StepState* st = a.st;
  if (MODE != 0 && st->done) return;
  const double dt = (MODE != 0) ? st->dt : 0.0;

  const Dims& d = a.d;
  const int t = threadIdx.x;
  const int ti0 = 1 + TI * (tile % a.ntile_i);
  const int tj0 = 1 + TJ * (tile / a.ntile_i);
  const int kb = 1 + a.kchunk * kc;
  const int ke = min(kb + a.kchunk, d.KM - 1);
  if (kb >= ke) return;
  const long VOL = d.VOL;
  // the ring holds exact stage-input values only when it is stored in FP64
  constexpr bool kExactRing = sizeof(S) == 8;

  const FluxConsts<R> C{(R)a.gamma, (R)a.gam1, (R)a.gam1_inv};

  // Face flux.  The hybrid kernel reads the sensor's decision byte of the face
  // (global face index e: i-faces, j-faces, k-faces in the reference's
  // Ep/Fp/Gp order): 0 = linear upwind-5, evaluated here; 1 = characteristic
  // WENO5, evaluated ahead of this kernel by the WENO5-face pass into a.wflux.
  // While the audit has set force_weno every face is a WENO5 face.
  const bool all_weno = HYB && st->force_weno;
  const long nfi = (long)(d.IM - 1) * (d.JM - 2) * (d.KM - 2);
  const long nfj = (long)(d.IM - 2) * (d.JM - 1) * (d.KM - 2);
  // wb: the face's decision when already loaded (0/1), -1 to read it here
  auto flux = [&](const auto& ld, R nx, R ny, R nz, long e, int wb, R out[5]) {
    if constexpr (HYB) {
      if (all_weno || (wb >= 0 ? wb != 0 : __ldg(a.mask + e) != 0)) {
        const float* w = a.wflux + 8 * e;
        const float4 v = __ldg(reinterpret_cast<const float4*>(w));
        out[0] = v.x;
        out[1] = v.y;
        out[2] = v.z;
        out[3] = v.w;
        out[4] = __ldg(w + 4);
      } else {
        face_flux_linear<R>(ld, nx, ny, nz, C, out);
      }
    } else {
      face_flux<R>(ld, nx, ny, nz, C, out);
    }
  };

  // The i-face (round A) and j-face (round B) of this thread: half-warps take
  // 16 faces of one row each, the two halves of a warp rows 8 apart, so that
  // their reads of a plane row (pitch 22 floats) start 16 banks apart: the
  // face rounds' shared-memory reads take 720 wavefronts per plane instead of
  // 1,104 with faces numbered row by row.  Round A: warps 0-6 take rows w and
  // w+8, faces 0..15; warp 7 row 7 and the fx = 16 face of rows 0..14.
  auto face_a = [&](int& fx, int& fy) -> bool {
    const int w = t >> 5, l = t & 31;
    if (w < 7) {
      fx = l & 15;
      fy = w + 8 * (l >> 4);
    } else if (l < 16) {
      fx = l;
      fy = 7;
    } else {
      fx = TI;
      fy = l - 16;
    }
    return fy < TJ;
  };
  auto face_b = [&](int& fx, int& fy) {
    fx = t & 15;
    fy = (t >> 5) + 8 * ((t >> 4) & 1);
  };

  // column owned by this thread
  const int cx = t % TI, cy = t / TI;
  const int ci = ti0 + cx, cj = tj0 + cy;
  const bool col_thread = t < NC;
  const bool col_valid = col_thread && ci <= d.IM - 2 && cj <= d.JM - 2;

  auto load_ring = [&](int kp) {
    if (col_thread) {
      S* dst = &sm.ring[(kp + 6) % 6][0][t];
      if (ci <= d.IM + 1 && cj <= d.JM + 1) {
        const long o = node_off(d, ci, cj, kp);
#pragma unroll
        for (int n = 0; n < NEQ; ++n) dst[n * NC] = (S)__ldg(a.src + n * VOL + o);
      }
    }
  };
  auto load_zeta = [&](int kp, double z[3]) {
    const long o = node_off(d, ci, cj, kp);
#pragma unroll
    for (int m = 0; m < 3; ++m) z[m] = __ldg(a.area[6 + m] + o);
  };

  // k-face between planes kk and kk+1 of this thread's column
  auto k_face = [&](int kk, const double za[3], const double zb[3], int wb, R out[5]) {
    const int s0 = (kk - 2 + 6) % 6;
    auto ld = [&](int p, int n) -> R {
      int s = s0 + p;
      s = s >= 6 ? s - 6 : s;
      return (R)sm.ring[s][n][t];
    };
    const long e = nfi + nfj + (ci - 1) + (long)(d.IM - 2) * ((cj - 1) + (long)(d.JM - 2) * kk);
    flux(ld, R(0.5) * ((R)za[0] + (R)zb[0]), R(0.5) * ((R)za[1] + (R)zb[1]), R(0.5) * ((R)za[2] + (R)zb[2]), e, wb,
         out);
  };

  // The FP32 kernels fetch the ring column of plane k+4 into registers while
  // plane k is computed and store it at the top of the next iteration, so the
  // ring load is off the critical path (the FP64 kernel has no registers to spare).
  constexpr bool kPrefetch = sizeof(S) == 4;
  double pre[NEQ];
  auto fetch_ring = [&](int kp) {
    if (col_thread && ci <= d.IM + 1 && cj <= d.JM + 1) {
      const long o = node_off(d, ci, cj, kp);
#pragma unroll
      for (int n = 0; n < NEQ; ++n) pre[n] = __ldg(a.src + n * VOL + o);
    }
  };
  auto store_ring = [&](int kp) {
    if (col_thread && ci <= d.IM + 1 && cj <= d.JM + 1) {
      S* dst = &sm.ring[(kp + 6) % 6][0][t];
#pragma unroll
      for (int n = 0; n < NEQ; ++n) dst[n * NC] = (S)pre[n];
    }
  };

  // halo node e of a plane: tile-relative (x, y)
  auto halo_xy = [&](int e, int& x, int& y) {
    if (e < NHI) {
      const int c6 = e % (2 * H);
      y = e / (2 * H);
      x = c6 < H ? c6 - H : TI + (c6 - H);
    } else {
      const int e2 = e - NHI;
      const int r6 = e2 / TI;
      x = e2 % TI;
      y = r6 < H ? r6 - H : TJ + (r6 - H);
    }
  };
  // TMA copies of plane kp's halo and face-node area vectors (area buffer
  // kp & 1), issued by thread 0 after a CTA barrier that ended every read of
  // the buffers they overwrite
  auto issue_plane = [&](int kp) {
    if constexpr (kTma) {
      if (t == 0) {
        unsigned long long* bar = &ts->bar[kp & 1];
        tma::fence_proxy();
        tma::bar_expect(bar, kTmaBytes);
        const int z = kp + NG, y0 = tj0 + NG;
        const int xl = (int)LP + NG + ti0 - 4, xc = (int)LP + NG + ti0, xr = (int)LP + NG + ti0 + TI;
        tma::load_4d(ts->hl, &tm->q_a, xl, y0, z, 0, bar);
        tma::load_4d(ts->hr, &tm->q_a, xr, y0, z, 0, bar);
        tma::load_4d(ts->hb, &tm->q_b, xc, y0 - H, z, 0, bar);
        tma::load_4d(ts->ht, &tm->q_b, xc, y0 + TJ, z, 0, bar);
        tma::load_4d(ts->area[kp & 1].xi, &tm->xi, xl, y0, z, 0, bar);
        tma::load_4d(ts->area[kp & 1].eta, &tm->eta, xc, y0 - 1, z, 3, bar);
      }
    }
  };

  // FP64 TMA kernel: the copies of plane kp's set -- its ring column three
  // planes ahead (kp+3), the plane with its halo, the area vectors -- on
  // barrier q & 1 (q = kp - kb + 1; the warm-up set is q = 0)
  auto issue_set64 = [&](int kp) {
    if constexpr (kTma64) {
      if (t == 0) {
        unsigned long long* bar = &t64->bar[(kp - kb + 1) & 1];
        tma::fence_proxy();
        tma::bar_expect(bar, kTma64Plane);
        const int z = kp + NG, y0 = tj0 + NG;
        const int xl = (int)LP + NG + ti0 - 4, xc = (int)LP + NG + ti0;
        tma::load_4d(&sm.ring[(kp + 3) % 6][0][0], &tm->q_a, xc, y0, kp + 3 + NG, 0, bar);
        tma::load_4d(&sm.plane[0][0][0], &tm->q_b, xl, y0 - H, z, 0, bar);
        tma::load_4d(&t64->xi[0][0][0], &tm->xi, xl, y0, z, 0, bar);
        tma::load_4d(&t64->eta[0][0][0], &tm->eta, xc, y0 - 1, z, 3, bar);
      }
    }
  };

  if constexpr (kTma || kTma64) {
    if (t == 0) {
      tma::bar_init(kTma ? &ts->bar[0] : &t64->bar[0]);
      tma::bar_init(kTma ? &ts->bar[1] : &t64->bar[1]);
      tma::fence_init();
    }
    __syncthreads();  // no thread waits on a barrier before it is initialised
  }
  // warm-up: planes kb-3 .. kb+2 and the kb-1/2 face
  bool landed = true;
  if constexpr (kTma64) {
    if (t == 0) {
      tma::bar_expect(&t64->bar[0], kTma64Warm);
      for (int kp = kb - 3; kp <= kb + 2; ++kp)
        tma::load_4d(&sm.ring[(kp + 6) % 6][0][0], &tm->q_a, (int)LP + NG + ti0, tj0 + NG, kp + NG, 0, &t64->bar[0]);
    }
  } else {
    for (int kp = kb - 3; kp <= kb + 2; ++kp) load_ring(kp);
  }
  if (kPrefetch) fetch_ring(kb + 3);
  if (kTma) issue_plane(kb);
  // the column's J*grad(zeta) at planes k and k+1, in FP64 (the stage-3
  // spectral radius uses it exactly)
  double za[3] = {0, 0, 0}, zb[3] = {0, 0, 0};
  if (col_valid) {
    load_zeta(kb - 1, za);
    load_zeta(kb, zb);
  }
  if constexpr (kTma64) landed = tma::bar_wait(&t64->bar[0], 0);
  if (__syncthreads_or(!landed)) {
    if (t == 0) {
      atomicExch(&a.st->stage_fail, 1);
      tma::bar_wait(&t64->bar[0], 0);  // bounded: the copies in flight
    }
    return;
  }
  R fkm[5] = {0, 0, 0, 0, 0};
  if (col_valid) k_face(kb - 1, za, zb, -1, fkm);
#pragma unroll
  for (int m = 0; m < 3; ++m) za[m] = zb[m];
  if constexpr (kTma64) {
    __syncthreads();  // the warm-up face has read the slot plane kb+3 lands in
    issue_set64(kb);
  }

  double smax = 0.0;  // running spectral-radius max (stage 3, inviscid)
  bool snan = false;

  // Hybrid: the decisions of this thread's i-, j- and k-face of plane k (bits
  // 0, 1, 2), read one plane ahead; the WENO5 fluxes of the set ones are
  // asked into L1 at the top of the plane, before the staging, so the face
  // rounds find them there.
  auto mask_bits = [&](int k) -> unsigned {
    unsigned m = 0;
    if constexpr (HYB) {
      int fx, fy;
      if (face_a(fx, fy)) {
        const int ga = ti0 + fx - 1, gj = tj0 + fy;
        if (ga <= d.IM - 2 && gj <= d.JM - 2)
          m |= __ldg(a.mask + ga + (long)(d.IM - 1) * ((gj - 1) + (long)(d.JM - 2) * (k - 1))) != 0;
      }
      {
        face_b(fx, fy);
        const int gi = ti0 + fx, ga = tj0 + fy - 1;
        if (gi <= d.IM - 2 && ga <= d.JM - 2)
          m |= (unsigned)(__ldg(a.mask + nfi + (gi - 1) + (long)(d.IM - 2) * (ga + (long)(d.JM - 1) * (k - 1))) != 0)
               << 1;
      }
      if (col_valid)
        m |= (unsigned)(__ldg(a.mask + nfi + nfj + (ci - 1) + (long)(d.IM - 2) * ((cj - 1) + (long)(d.JM - 2) * k)) !=
                        0)
             << 2;
    }
    return m;
  };
  auto prefetch_weno = [&](int k, unsigned m) {
    if constexpr (HYB) {
      int fx, fy;
      if (m & 1u) {
        face_a(fx, fy);
        const int ga = ti0 + fx - 1, gj = tj0 + fy;
        prefetch_l1(a.wflux + 8 * (ga + (long)(d.IM - 1) * ((gj - 1) + (long)(d.JM - 2) * (k - 1))));
      }
      if (m & 2u) {
        face_b(fx, fy);
        const int gi = ti0 + fx, ga = tj0 + fy - 1;
        prefetch_l1(a.wflux + 8 * (nfi + (gi - 1) + (long)(d.IM - 2) * (ga + (long)(d.JM - 1) * (k - 1))));
      }
      if (m & 4u) prefetch_l1(a.wflux + 8 * (nfi + nfj + (ci - 1) + (long)(d.IM - 2) * ((cj - 1) + (long)(d.JM - 2) * k)));
    }
  };
  unsigned mnext = (HYB && !all_weno) ? mask_bits(kb) : 0u;

  for (int k = kb; k < ke; ++k) {
    if (col_valid) load_zeta(k + 1, zb);  // consumed in round C
    const unsigned mcur = mnext;
    if constexpr (HYB) {
      if (!all_weno) {
        prefetch_weno(k, mcur);
        if (k + 1 < ke) mnext = mask_bits(k + 1);
      }
    }
    // viscous kernels ask L2 for the next plane's viscous divergence
    if (VISC && MODE != 0 && col_valid && k + 1 < ke) {
      const long o = node_off(d, ci, cj, k + 1);
#pragma unroll
      for (int n = 0; n < 4; ++n) prefetch_l2(reinterpret_cast<const AreaT<R>*>(a.dfv[n]) + o);
    }
    // the FP32 kernels ask L2 for the next plane's RK operands and 1/J now, so
    // the update's loads one plane later find them there
    if (sizeof(S) == 4 && MODE != 0 && col_valid && k + 1 < ke) {
      const long o = node_off(d, ci, cj, k + 1);
      prefetch_l2(a.area[9] + o);
#pragma unroll
      for (int n = 0; n < NEQ; ++n) {
        prefetch_l2(a.q0 + n * VOL + o);
        if (MODE >= 2) prefetch_l2(a.qp + n * VOL + o);
      }
    }
    // plane k's halo and area vectors (FP32 TMA kernels), plane k's set (FP64
    // TMA kernel) have landed; a wait that runs out on any thread ends the
    // CTA's work, recorded in st->stage_fail
    unsigned long long* wbar = nullptr;
    unsigned wpar = 0;
    if constexpr (kTma) {
      wbar = &ts->bar[k & 1];
      wpar = ((k - kb) >> 1) & 1;
    } else if constexpr (kTma64) {
      wbar = &t64->bar[(k - kb + 1) & 1];
      wpar = ((k - kb + 1) >> 1) & 1;
    }
    if constexpr (kTma || kTma64) landed = tma::bar_wait(wbar, wpar);
    if (__syncthreads_or(!landed)) {
      if (t == 0) {
        atomicExch(&a.st->stage_fail, 1);
        tma::bar_wait(wbar, wpar);  // bounded: the copies in flight
      }
      return;
    }
    if constexpr (kTma64) {
      // ring column, plane and area vectors are in place
    } else if (kPrefetch) {
      store_ring(k + 3);
      if (k + 1 < ke) fetch_ring(k + 4);
    } else {
      load_ring(k + 3);
    }
    // plane k with halo: interior from the ring, halo from global memory
    if constexpr (!kTma64) {
      const int sk = k % 6;
      for (int e = t; e < NC; e += NT) {
        const int x = e % TI, y = e / TI;
#pragma unroll
        for (int n = 0; n < NEQ; ++n) sm.plane[n][y + H][x + H] = sm.ring[sk][n][e];
      }
      // halo: 6 columns x TJ rows (i-halo) then 6 rows x TI columns (j-halo)
      for (int e = t; e < NHI + NHJ; e += NT) {
        int x, y;
        halo_xy(e, x, y);
        const int gi = ti0 + x, gj = tj0 + y;
        if (gi <= d.IM + 1 && gj <= d.JM + 1) {
          if (kTma) {
#pragma unroll
            for (int n = 0; n < NEQ; ++n)
              sm.plane[n][y + H][x + H] = (S)(x < 0 ? ts->hl[n][y][x + 4]
                                                     : x >= TI ? ts->hr[n][y][x - TI]
                                                               : y < 0 ? ts->hb[n][y + H][x] : ts->ht[n][y - TJ][x]);
          } else {
            const long o = node_off(d, gi, gj, k);
#pragma unroll
            for (int n = 0; n < NEQ; ++n) sm.plane[n][y + H][x + H] = (S)__ldg(a.src + n * VOL + o);
          }
        }
      }
      // area vectors of the face nodes of plane k (synchronous kernels)
      for (int e = t; !kTma && e < NSX + NSY; e += NT) {
        if (e < NSX) {
          const int c = e % (TI + 2), r = e / (TI + 2);
          const int gi = ti0 - 1 + c, gj = tj0 + r;
          if (gi <= d.IM + 1 && gj <= d.JM + 1) {
            const long o = node_off(d, gi, gj, k);
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              if constexpr (sizeof(R) == 4) asy->sx[m][r][c] = __ldg(a.area32[m] + o);
              else asy->sx[m][r][c] = __ldg(a.area[m] + o);
            }
          }
        } else {
          const int e2 = e - NSX;
          const int c = e2 % TI, r = e2 / TI;
          const int gi = ti0 + c, gj = tj0 - 1 + r;
          if (gi <= d.IM + 1 && gj <= d.JM + 1) {
            const long o = node_off(d, gi, gj, k);
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              if constexpr (sizeof(R) == 4) asy->sy[m][r][c] = __ldg(a.area32[3 + m] + o);
              else asy->sy[m][r][c] = __ldg(a.area[3 + m] + o);
            }
          }
        }
      }
    }
    if constexpr (!kTma64) __syncthreads();
    // plane k+1's halo and area vectors travel while plane k is computed (the
    // buffers they overwrite were last read by plane k-1 and by the staging)
    if (kTma && k + 1 < ke) issue_plane(k + 1);
    // the area vectors of plane k's face nodes: node (i0-1+c, j0+r) and (i0+c, j0-1+r)
    auto ax = [&](int m, int r, int c) -> R {
      if constexpr (kTma) return (R)ts->area[k & 1].xi[m][r][c + 3];
      else if constexpr (kTma64) return (R)t64->xi[m][r][c + 3];
      else return (R)asy->sx[m][r][c];
    };
    auto ay = [&](int m, int r, int c) -> R {
      if constexpr (kTma) return (R)ts->area[k & 1].eta[m][r][c];
      else if constexpr (kTma64) return (R)t64->eta[m][r][c];
      else return (R)asy->sy[m][r][c];
    };

    R fkp[5];
    // round A: i-faces.  Face fx (0..TI) of row fy lies between tile columns fx-1 and fx.
    int fx, fy;
    if (face_a(fx, fy)) {
      const int ga = ti0 + fx - 1, gj = tj0 + fy;
      if (ga <= d.IM - 2 && gj <= d.JM - 2) {
        auto ld = [&](int p, int n) -> R { return (R)sm.plane[n][fy + H][fx + p + X0]; };
        R f[5];
        const long e = ga + (long)(d.IM - 1) * ((gj - 1) + (long)(d.JM - 2) * (k - 1));
        flux(ld, R(0.5) * (ax(0, fy, fx) + ax(0, fy, fx + 1)), R(0.5) * (ax(1, fy, fx) + ax(1, fy, fx + 1)),
             R(0.5) * (ax(2, fy, fx) + ax(2, fy, fx + 1)), e, HYB ? (int)(mcur & 1u) : 0, f);
#pragma unroll
        for (int n = 0; n < NEQ; ++n) sm.fi[n][fy][fx] = f[n];
      }
    }
    // round B: j-faces.  Face fy (0..TJ) of column fx lies between tile rows fy-1 and fy.
    {
      face_b(fx, fy);
      const int gi = ti0 + fx, ga = tj0 + fy - 1;
      if (gi <= d.IM - 2 && ga <= d.JM - 2) {
        auto ld = [&](int p, int n) -> R { return (R)sm.plane[n][fy + p][fx + H + X0]; };
        R f[5];
        const long e = nfi + (gi - 1) + (long)(d.IM - 2) * (ga + (long)(d.JM - 1) * (k - 1));
        flux(ld, R(0.5) * (ay(0, fy, fx) + ay(0, fy + 1, fx)), R(0.5) * (ay(1, fy, fx) + ay(1, fy + 1, fx)),
             R(0.5) * (ay(2, fy, fx) + ay(2, fy + 1, fx)), e, HYB ? (int)((mcur >> 1) & 1u) : 0, f);
#pragma unroll
        for (int n = 0; n < NEQ; ++n) sm.fj[n][fy][fx] = f[n];
      }
    }
    // round C: the k+1/2 face of this column
    if (col_valid) k_face(k, za, zb, HYB ? (int)((mcur >> 2) & 1u) : 0, fkp);
    // The FP32 kernels built for 2 CTAs per SM issue part of the update's
    // loads (the RK base and 1/J) before the barrier, so that their latency
    // overlaps the wait for the other threads' flux rounds (split path 1.5%
    // faster on the bench grid); at 3 CTAs per SM (80 registers) the held
    // values spill and the kernel is 5% slower, so those load after it.
    constexpr bool kEarly = sizeof(S) == 4 && NB == 2;
    double pq0[NEQ], piJ = 0.0;
    if (kEarly && MODE != 0 && col_valid) {
      const long o = node_off(d, ci, cj, k);
      piJ = __ldg(a.area[9] + o);
#pragma unroll
      for (int n = 0; n < NEQ; ++n) pq0[n] = MODE == 3 ? a.q0[n * VOL + o] : __ldg(a.q0 + n * VOL + o);
    }
    __syncthreads();
    // FP64 TMA kernel: plane k+1's set travels during the update (it
    // overwrites the plane, the area vectors and plane k-2's ring slot, which
    // the rounds above were the last to read)
    if (kTma64 && k + 1 < ke) issue_set64(k + 1);

    if (col_valid) {
      const long o = node_off(d, ci, cj, k);
      double df[NEQ];
#pragma unroll
      for (int n = 0; n < NEQ; ++n)
        df[n] = (double)(sm.fi[n][cy][cx + 1] - sm.fi[n][cy][cx]) + (double)(sm.fj[n][cy + 1][cx] - sm.fj[n][cy][cx]) +
                (double)(fkp[n] - fkm[n]);
      if (VISC) {
        // the viscous flux divergence, formed by visc_div_kernel (visc.cu)
#pragma unroll
        for (int n = 0; n < 4; ++n) df[n + 1] -= (double)__ldg(reinterpret_cast<const AreaT<R>*>(a.dfv[n]) + o);
      }
      const double iJ = (kEarly && MODE != 0) ? piJ : __ldg(a.area[9] + o);
      if (MODE == 0) {
        const long r = 5L * ((ci - 1) + (long)(d.IM - 2) * ((cj - 1) + (long)(d.JM - 2) * (k - 1)));
#pragma unroll
        for (int n = 0; n < NEQ; ++n) a.out[r + n] = df[n] * iJ;
      } else {
        const int sk = k % 6;
        double q[NEQ];
#pragma unroll
        for (int n = 0; n < NEQ; ++n) {
          const double L = dt * (df[n] * iJ);
          const long e = n * VOL + o;
          const double qin = kExactRing ? (double)sm.ring[sk][n][t] : 0.0;
          const double q0v = kEarly ? pq0[n] : (MODE == 3 ? a.q0[e] : __ldg(a.q0 + e));
          const double qpv = MODE >= 2 ? __ldg(a.qp + e) : 0.0;
          if (MODE == 1) {
            q[n] = ((kExactRing && a.q0_is_src) ? qin : q0v) - L;
          } else if (MODE == 2) {
            q[n] = 0.75 * q0v + 0.25 * (((kExactRing && a.qp_is_src) ? qin : qpv) - L);
          } else {
            // the plain (FP64) kernel divides by 3 as the reference does; the
            // FP32-flux kernels multiply by the rounded 1/3 (one ulp apart)
            const double sum = q0v + 2.0 * (((kExactRing && a.qp_is_src) ? qin : qpv) - L);
            q[n] = kExactRing ? sum / 3.0 : sum * (1.0 / 3.0);
          }
        }
#pragma unroll
        for (int n = 0; n < NEQ; ++n) a.out[n * VOL + o] = q[n];
        if (VISC || a.sigma) {
          const double r = q[0], ir = __drcp_rn(r);
          const double uu = __dmul_rn(q[1], ir), vv = __dmul_rn(q[2], ir), ww = __dmul_rn(q[3], ir);
          const double ke = __fma_rn(ww, ww, __fma_rn(vv, vv, __dmul_rn(uu, uu)));
          const double pp = __dmul_rn(a.gam1, __fma_rn(-__dmul_rn(0.5, r), ke, q[4]));
          if (VISC) {
            a.prim[0][o] = r;
            a.prim[1][o] = uu;
            a.prim[2][o] = vv;
            a.prim[3][o] = ww;
            a.prim[4][o] = pp;
            a.prim[5][o] = a.gM2 * pp / r;
          } else {
            // grad(xi), grad(eta), grad(zeta) = area vectors / J, the spectral
            // radius in FP64: xi and eta from the plane's staged face-node
            // area vectors (FP64 in the plain kernel; the FP32 kernels' FP32
            // copies, as their fluxes use them, which moves dt by ~1e-7
            // relative and spares 48 B per node of stage 3's loads), from
            // memory in the FP64 TMA kernel (its staging is being refilled);
            // zeta from the registers
            double g[9];
#pragma unroll
            for (int m = 0; m < 3; ++m) {
              if constexpr (kTma64) {
                g[m] = __dmul_rn(__ldg(a.area[m] + o), iJ);
                g[3 + m] = __dmul_rn(__ldg(a.area[3 + m] + o), iJ);
              } else {
                g[m] = __dmul_rn((double)ax(m, cy, cx + 1), iJ);
                g[3 + m] = __dmul_rn((double)ay(m, cy + 1, cx), iJ);
              }
              g[6 + m] = __dmul_rn(za[m], iJ);
            }
            // explicit roundings: every compilation of this kernel (single
            // and batched) then gives the same dt to the last bit
            const double cs = __dsqrt_rn(__ddiv_rn(__dmul_rn(a.gamma, pp), r));
            double s = 0.0;
#pragma unroll
            for (int dd = 0; dd < 3; ++dd) {
              const double mx = g[3 * dd], my = g[3 * dd + 1], mz = g[3 * dd + 2];
              const double un = __fma_rn(ww, mz, __fma_rn(vv, my, __dmul_rn(uu, mx)));
              const double nn = __fma_rn(mz, mz, __fma_rn(my, my, __dmul_rn(mx, mx)));
              s = __dadd_rn(s, __dadd_rn(fabs(un), __dmul_rn(cs, __dsqrt_rn(nn))));
            }
            if (s != s) snan = true;
            smax = fmax(smax, s);
          }
        }
      }
    }
#pragma unroll
    for (int n = 0; n < NEQ; ++n) fkm[n] = fkp[n];
#pragma unroll
    for (int m = 0; m < 3; ++m) za[m] = zb[m];
  }

  if constexpr (kTma || kTma64) {
    // every issued copy was waited for: nothing is in flight; retire the
    // barriers so a batched CTA can initialise them again for its next item
    __syncthreads();
    if (t == 0) {
      tma::bar_inval(kTma ? &ts->bar[0] : &t64->bar[0]);
      tma::bar_inval(kTma ? &ts->bar[1] : &t64->bar[1]);
    }
  }
  if (MODE != 0 && !VISC && a.sigma) {
    // CTA max, one atomic per CTA
    __shared__ double red[NT / 32];
    __shared__ int rnan;
    if (t == 0) rnan = 0;
    double m = smax;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, s));
    __syncthreads();
    if (snan) rnan = 1;
    if ((t & 31) == 0) red[t >> 5] = m;
    __syncthreads();
    if (t == 0) {
      for (int w = 1; w < NT / 32; ++w) m = fmax(m, red[w]);
      atomic_max_sigma(&a.st->sigma_bits, rnan ? __longlong_as_double(0x7ff8000000000000ll) : m);
    }
  }
}

template <typename R, bool VISC, int MODE, int NB, bool HYB, bool TMA>
__global__ void __launch_bounds__(NT, NB) stage_kernel(const __grid_constant__ StageArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  stage_body<R, VISC, MODE, NB, HYB, TMA>(a, &a.tm, blockIdx.x, blockIdx.y, smem_raw);
}

// Many blocks in one launch: persistent CTAs take work items (block, tile, k
// chunk) from a queue (one atomic counter); each item's StageArgs are copied
// from the table into shared memory.  Items are numbered block by block, tiles
// fastest, so CTAs of one block work on neighbouring columns together.  The
// TMA copies read their tensor maps from the table in global memory.
template <typename R, bool VISC, int MODE, int NB, bool HYB, bool TMA>
__global__ void __launch_bounds__(NT, NB) stage_kernel_batched(const BatchStage b) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ StageArgs args;
  __shared__ int item;
  for (;;) {
    if (threadIdx.x == 0) item = (int)atomicAdd(b.counter, 1u);
    __syncthreads();
    const int w = item;
    if (w >= b.total) break;
    int blk = 0;
    while (blk + 1 < b.nblocks && __ldg(b.start + blk + 1) <= w) ++blk;
    const int* src = reinterpret_cast<const int*>(b.args + blk);
    int* dst = reinterpret_cast<int*>(&args);
    for (int e = threadIdx.x; e < (int)(sizeof(StageArgs) / sizeof(int)); e += NT) dst[e] = __ldg(src + e);
    __syncthreads();
    const int local = w - __ldg(b.start + blk);
    const int ntiles = args.ntile_i * args.ntile_j;
    stage_body<R, VISC, MODE, NB, HYB, TMA>(args, &b.args[blk].tm, local % ntiles, local / ntiles, smem_raw);
    __syncthreads();  // args, item and the shared staging are reused by the next item
  }
}


// The batched kernels run at 2 CTAs per SM (3 for the hybrid, whose stage
// kernel holds no WENO5 code); the FP32 ones stage by TMA, the FP64 one
// synchronously (its TMA form leaves no room for the item's StageArgs).
template <bool HYB>
constexpr int batched_nb() {
  return HYB ? 3 : 2;
}

template <typename R, bool VISC, int MODE, bool HYB>
cudaError_t launch_batched_t(const BatchStage& b, cudaStream_t s) {
  constexpr int NB = batched_nb<HYB>();
  constexpr bool TMA = sizeof(R) == 4;
  const int smem = (int)stage_smem<R, NB, TMA>();
  static int grid = 0;
  if (grid == 0) {
    cudaError_t e = cudaFuncSetAttribute(stage_kernel_batched<R, VISC, MODE, NB, HYB, TMA>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(stage_kernel_batched<R, VISC, MODE, NB, HYB, TMA>,
                               cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    int per_sm = 0, dev = 0, nsm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, stage_kernel_batched<R, VISC, MODE, NB, HYB, TMA>, NT,
                                                      smem);
    if (e == cudaSuccess) e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    grid = nsm * (per_sm > 0 ? per_sm : 1);
  }
  const int g = b.total < grid ? b.total : grid;
  if (g <= 0) return cudaSuccess;
  stage_kernel_batched<R, VISC, MODE, NB, HYB, TMA><<<g, NT, smem, s>>>(b);
  return cudaGetLastError();
}

template <typename R, bool HYB>
cudaError_t launch_batched_r(const BatchStage& b, int mode, bool visc, cudaStream_t s) {
  if (visc) {
    switch (mode) {
      case 1: return launch_batched_t<R, true, 1, HYB>(b, s);
      case 2: return launch_batched_t<R, true, 2, HYB>(b, s);
      default: return launch_batched_t<R, true, 3, HYB>(b, s);
    }
  }
  switch (mode) {
    case 1: return launch_batched_t<R, false, 1, HYB>(b, s);
    case 2: return launch_batched_t<R, false, 2, HYB>(b, s);
    default: return launch_batched_t<R, false, 3, HYB>(b, s);
  }
}

template <typename R, bool VISC, int MODE, int NB, bool HYB, bool TMA>
cudaError_t launch_t(const StageArgs& a, cudaStream_t s) {
  const size_t smem = stage_smem<R, NB, TMA>();
  dim3 grid(a.ntile_i * a.ntile_j, (a.d.KM - 2 + a.kchunk - 1) / a.kchunk);
  stage_kernel<R, VISC, MODE, NB, HYB, TMA><<<grid, NT, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename R, int NB, bool HYB, bool TMA>
void prepare_nb() {
  const int smem = (int)stage_smem<R, NB, TMA>();
  // the largest shared-memory carveout, so that NB CTAs fit on an SM
  auto set = [&](const void* f) {
    cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
  };
  set((const void*)stage_kernel<R, false, 0, NB, HYB, TMA>);
  set((const void*)stage_kernel<R, false, 1, NB, HYB, TMA>);
  set((const void*)stage_kernel<R, false, 2, NB, HYB, TMA>);
  set((const void*)stage_kernel<R, false, 3, NB, HYB, TMA>);
  set((const void*)stage_kernel<R, true, 0, NB, HYB, TMA>);
  set((const void*)stage_kernel<R, true, 1, NB, HYB, TMA>);
  set((const void*)stage_kernel<R, true, 2, NB, HYB, TMA>);
  set((const void*)stage_kernel<R, true, 3, NB, HYB, TMA>);
}

template <typename R, int NB, bool HYB, bool TMA>
cudaError_t launch_r(const StageArgs& a, int mode, bool visc, cudaStream_t s) {
  if (visc) {
    switch (mode) {
      case 0: return launch_t<R, true, 0, NB, HYB, TMA>(a, s);
      case 1: return launch_t<R, true, 1, NB, HYB, TMA>(a, s);
      case 2: return launch_t<R, true, 2, NB, HYB, TMA>(a, s);
      default: return launch_t<R, true, 3, NB, HYB, TMA>(a, s);
    }
  }
  switch (mode) {
    case 0: return launch_t<R, false, 0, NB, HYB, TMA>(a, s);
    case 1: return launch_t<R, false, 1, NB, HYB, TMA>(a, s);
    case 2: return launch_t<R, false, 2, NB, HYB, TMA>(a, s);
    default: return launch_t<R, false, 3, NB, HYB, TMA>(a, s);
  }
}

}  // namespace

// Raise the dynamic shared-memory limit of every instantiation once (outside
// any stream capture).
void stage_prepare() {
  static bool done = false;
  if (done) return;
  prepare_nb<double, 2, false, false>();
  prepare_nb<double, 2, false, true>();
  prepare_nb<float, 2, false, true>();
  prepare_nb<float, 3, false, true>();
  prepare_nb<float, 2, true, true>();
  prepare_nb<float, 3, true, true>();
  prepare_nb<float, 4, true, false>();
  done = true;
}

void stage_tiles(const Dims& d, int* ntile_i, int* ntile_j) {
  *ntile_i = (d.IM - 2 + TI - 1) / TI;
  *ntile_j = (d.JM - 2 + TJ - 1) / TJ;
}

// FP64: 2 CTAs per SM, synchronous (variant 0) or TMA staging (variant 1);
// split FP32: 2 or 3 CTAs per SM; hybrid: 2, 3 or 4 (FP32 variant = CTAs per
// SM - 2; TMA staging at 2 and 3).
int stage_variants(bool fp32, bool hybrid) { return !fp32 ? 2 : (hybrid ? 3 : 2); }

cudaError_t launch_stage_batched(const BatchStage& b, int mode, bool visc, bool fp32, bool hybrid, cudaStream_t s) {
  if (mode < 1 || mode > 3) return cudaErrorInvalidValue;
  if (!fp32) return launch_batched_r<double, false>(b, mode, visc, s);
  if (hybrid) return launch_batched_r<float, true>(b, mode, visc, s);
  return launch_batched_r<float, false>(b, mode, visc, s);
}

cudaError_t launch_stage(const StageArgs& a, int mode, bool visc, bool fp32, int variant, cudaStream_t s) {
  if (!fp32)
    return variant == 1 ? launch_r<double, 2, false, true>(a, mode, visc, s)
                        : launch_r<double, 2, false, false>(a, mode, visc, s);
  if (a.mask) {
    if (variant == 2) return launch_r<float, 4, true, false>(a, mode, visc, s);
    return variant == 1 ? launch_r<float, 3, true, true>(a, mode, visc, s)
                        : launch_r<float, 2, true, true>(a, mode, visc, s);
  }
  return variant == 1 ? launch_r<float, 3, false, true>(a, mode, visc, s)
                      : launch_r<float, 2, false, true>(a, mode, visc, s);
}

}  // namespace cbns
