// adjoint.cu -- reverse-mode gradients of a velocity-Verlet trajectory.
//
// Forward step n -> n+1 as the engine runs it (Berendsen scale lambda_n is
// applied lazily by the next step's first kernel):
//   u      = lambda_n v_n + (dt/2m) F(x_n)
//   x_n+1  = x_n + dt u
//   v_n+1  = u + (dt/2m) F(x_n+1)
//   K_n+1  = 1/2 sum m v_n+1^2,  lambda_n+1 = g(K_n+1)
//          = sqrt(max(0, 1 + dt/tau (kT0 dof / (2 K) - 1)))
// with observables PE(x_n), W(x_n) (virial sum r.F) and KE_n = lambda_n^2 K_n.
//
// Walking back over step m (m = T .. 0), with u_bar_m+1 the adjoint of the
// next step's pre-kick velocity (0 after the last step):
//   K_bar = g_KE lambda^2 + (sum u_bar_m+1 . v_m + g_KE 2 lambda K) g'(K)
//   v_bar = lambda u_bar_m+1 + K_bar m v_m
//   F_bar = (dt/2m) (u_bar_m+1 + v_bar)        (m = 0: (dt/2m) u_bar_1)
//   x_bar += g_PE grad PE + g_W grad W + J(x_m) F_bar,  J = dF/dx (symmetric)
//   u_bar_m = v_bar + dt x_bar
// and the parameter adjoints collect F_bar . dF/dtheta + g_PE dPE/dtheta +
// g_W dW/dtheta.  For a pair with d = x_i - x_j and phi = F_ij / d (so that
// F_i = sum_j phi d), A_ij = phi I + (phi'/r) d d^T and
//   (J F_bar)_i = sum_j A_ij (F_bar_i - F_bar_j)
// over the full neighbour list: every particle gathers, no atomics.
//
// The neighbour list of each replayed step is the one the forward step used:
// it is rebuilt (deterministically, slots never reorder during an adjoint
// run) from the positions of that step's last build.
#include "adjoint.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "bonded_math.cuh"
#include "device_util.cuh"
#include "engine.hpp"
#include "kernels.cuh"
#include "trace.hpp"

namespace bb {

AdjointStore::~AdjointStore() {
  for (void* p : allocations) cudaFree(p);
}

template <typename T>
T* AdjointStore::alloc(size_t count) {
  void* p = nullptr;
  cuda_check(cudaMalloc(&p, std::max<size_t>(1, count) * sizeof(T)), "cudaMalloc (adjoint)");
  allocations.push_back(p);
  cuda_check(cudaMemsetAsync(p, 0, std::max<size_t>(1, count) * sizeof(T), stream),
             "cudaMemset (adjoint)");
  return static_cast<T*>(p);
}

namespace {

constexpr int kAdjTypes = 4;  // largest LJ table side the adjoint supports

// Device view of the adjoint store.
struct AdjView {
  float4* seg_pos;
  float4* seg_vel;
  const double* seg_lam;
  const double* seg_kin;
  float4* xbar;
  float4* vbar;
  float4* fbar;
  float4* ubar;
  const double* obs_grad;
  long long* theta;
  const float4* ck_ref_pos;
  const int* list_src;   // per replica: -1 checkpoint build positions, else step index
  const uint32_t* snap_nbr;  // list snapshots (null: the current list, rebuilt per step)
  const uint32_t* snap_cnt;
  uint64_t snap_entries;     // list entries per snapshot
  const int* shift_on;   // per replica: LJ energy shift active
  long long* dot;        // [2 lanes][R][whole, frac]: sum u_bar . v, double-buffered
  long long* theta_bond;      // [global bond type][k, r0][whole, frac]
  long long* theta_angle;     // [global angle type][k, theta0 (rad)][whole, frac]
  long long* theta_dihedral;  // [global dihedral type][k][whole, frac]
  uint32_t slots;
  uint32_t replicas;
};

__global__ void k_adj_record(DeviceView v, double* lam, double* kin, uint32_t* flags,
                             uint32_t k) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= v.n_replicas) return;
  const ReplicaState& st = v.rs[r];
  lam[(size_t)k * v.n_replicas + r] = st.lambda;
  kin[(size_t)k * v.n_replicas + r] = st.last_kinetic;
  flags[(size_t)k * v.n_replicas + r] = st.need_rebuild;
}

// Positions from which each replica's list of the current replayed step was
// built, and the rebuild flags for the replicas whose list changes.
__global__ void k_adj_list_positions(DeviceView v, AdjView a, uint32_t segment,
                                     const uint32_t* changed) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const uint32_t i = b * kBlock + threadIdx.x;
  if (threadIdx.x == 0 && (i - v.rp[r].atom_begin) == 0u) {
    v.rs[r].need_rebuild = changed[r];
    v.rs[r].reorder_now = 0u;
  }
  if (!changed[r]) return;
  const int src = a.list_src[r];
  v.pos[i] = src < 0 ? a.ck_ref_pos[(size_t)segment * a.slots + i]
                     : a.seg_pos[(size_t)src * a.slots + i];
}

// Copies the list rows (and counts) of slot block b into snapshot k: every
// block when `all`, else the blocks of replicas that rebuilt their list in
// the step just run.  A block's 128 rows are one contiguous run of the
// interleaved list (4 whole groups of 32 rows).
__global__ void k_adj_snapshot(DeviceView v, uint32_t* snap_nbr, uint32_t* snap_cnt,
                               uint32_t k, int all) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  if (!all && !v.rs[r].need_rebuild) return;
  const size_t entries = (size_t)kBlock * v.nbr_stride;
  const size_t base = (size_t)b * entries;
  const size_t per_snap = (size_t)v.n_slots * v.nbr_stride;
  const uint4* src = reinterpret_cast<const uint4*>(v.nbr + base);
  uint4* dst = reinterpret_cast<uint4*>(snap_nbr + (size_t)k * per_snap + base);
  for (size_t t = threadIdx.x; t < entries / 4; t += blockDim.x) dst[t] = __ldcs(src + t);
  if (threadIdx.x < kBlock) {
    const size_t i = (size_t)b * kBlock + threadIdx.x;
    snap_cnt[(size_t)k * v.n_slots + i] = v.nbr_count[i];
  }
}

// Crossing counts of restored slots: img - ref_img of the checkpoint.
__global__ void k_adj_cross(DeviceView v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.n_slots) return;
  const int4 im = v.img[i], ri = v.ref_img[i];
  v.cross[i] = pack_cross(im.x - ri.x, im.y - ri.y, im.z - ri.z);
}

__global__ void k_adj_mark_all(DeviceView v) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= v.n_replicas) return;
  v.rs[r].need_rebuild = 1u;
  v.rs[r].reorder_now = 0u;
}

// Step m, part 1: kinetic-energy and Berendsen adjoints, v_bar, F_bar.
// Reads the sum u_bar_m+1 . v_m from lane `lane_in` of a.dot (written by the
// pair kernel of step m+1) and clears it in its last block.
__global__ void __launch_bounds__(kBlock)
k_adj_prepare(DeviceView v, AdjView a, uint32_t m, uint32_t k, int first, int last,
              int lane_in) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  const uint32_t i = b * kBlock + threadIdx.x;
  const bool real = (i - p.atom_begin) < p.n_atoms;
  const double lam = a.seg_lam[(size_t)k * v.n_replicas + r];
  const double kin = a.seg_kin[(size_t)k * v.n_replicas + r];
  const double g_ke = a.obs_grad[((size_t)m * v.n_replicas + r) * 3 + 2];
  long long* din = a.dot + ((size_t)lane_in * v.n_replicas + r) * 2;
  const double dot = last ? 0.0 : from_fixed(din[0], din[1]);
  double gp = 0.0;
  if (!first && p.thermostat == 1 && kin > 0.0 && p.dof > 0.0 && lam > 0.0) {
    const double c = (double)p.dt / p.tau;
    const double big_a = 0.5 * p.kt_target * p.dof;
    gp = c * (-big_a / (kin * kin)) / (2.0 * lam);
  }
  const double k_bar = g_ke * lam * lam + (dot + g_ke * 2.0 * lam * kin) * gp;
  if (real) {
    const float4 vel = a.seg_vel[(size_t)k * a.slots + i];
    const float4 u = last ? make_float4(0.f, 0.f, 0.f, 0.f) : a.ubar[i];
    const float l = (float)lam;
    const float km = (float)(k_bar * (double)vel.w);
    float4 vb;
    vb.x = __fmaf_rn(l, u.x, km * vel.x);
    vb.y = __fmaf_rn(l, u.y, km * vel.y);
    vb.z = __fmaf_rn(l, u.z, km * vel.z);
    vb.w = 0.f;
    const float h = __fdiv_rn(__fmul_rn(0.5f, p.dt), vel.w);
    float4 fb;
    if (first) {
      fb = make_float4(h * u.x, h * u.y, h * u.z, 0.f);
    } else {
      fb = make_float4(h * (u.x + vb.x), h * (u.y + vb.y), h * (u.z + vb.z), 0.f);
    }
    a.vbar[i] = vb;
    a.fbar[i] = fb;
  }
  const uint32_t n_blocks = p.n_pad / kBlock;
  if (arrive_last(&st->done_post, n_blocks) && threadIdx.x == 0) {
    din[0] = 0;
    din[1] = 0;
    st->done_post = 0u;
  }
}

// Per type pair constants of the adjoint pair kernel.
struct AdjCoeff {
  float sigma2, eps4, eps24, shift;
  float inv_eps;  // 1/eps (0 when eps = 0: the eps derivative is then 0)
  float inv_sig;  // 1/sigma
  float dshift;   // d(energy shift)/d(sigma)
  float pad;
};

template <int kNt>
__device__ __forceinline__ void add_typed(float (&acc)[kNt], int t, float v) {
#pragma unroll
  for (int c = 0; c < kNt; ++c) acc[c] += (c == t) ? v : 0.0f;
}

// Step m, part 2: x_bar += g_PE grad PE + g_W grad W + J F_bar over the LJ
// pairs, parameter adjoints, then u_bar_m and the sum u_bar_m . v_m-1 (lane
// `lane_out` of a.dot).  `pos` holds x_m.  Batches of four list entries with
// the next batch's entries requested early, as in the force kernel; kNt is
// the LJ table side rounded up (2 or 4).
template <int kNt, int kTpa>
__global__ void __launch_bounds__(kBlock)
k_adj_lj(DeviceView v, AdjView a, const float4* __restrict__ pos, uint32_t m, uint32_t k,
         int first, int lane_out, int finish) {
  constexpr uint32_t kAtoms = kBlock / kTpa;
  const uint32_t b = blockIdx.x / kTpa;  // 128-slot block of the particles
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  __shared__ AdjCoeff table[kNt * kNt];
  __shared__ unsigned long long theta_sh[kAdjTypes * kAdjTypes * 2 * 2];
  const int nt = p.n_types;
  const float rc2 = p.force_cut_sq;
  const bool shift_on = a.shift_on[r] != 0;
  for (int t = threadIdx.x; t < nt * nt; t += kBlock) {
    const LjCoeff c = v.lj[p.lj_offset + t];
    AdjCoeff q;
    q.sigma2 = c.sigma2;
    q.eps4 = c.eps4;
    q.eps24 = c.eps24;
    q.shift = c.shift;
    q.inv_eps = c.eps4 != 0.0f ? 4.0f / c.eps4 : 0.0f;
    const float sig = sqrtf(c.sigma2);
    q.inv_sig = 1.0f / sig;
    q.dshift = 0.0f;
    if (shift_on) {
      const float sc2 = c.sigma2 / rc2;
      const float sc6 = sc2 * sc2 * sc2;
      q.dshift = c.eps4 * (12.0f * sc6 * sc6 - 6.0f * sc6) / sig;
    }
    q.pad = 0.0f;
    table[(t / nt) * kNt + (t % nt)] = q;
  }
  for (int t = threadIdx.x; t < kAdjTypes * kAdjTypes * 4; t += kBlock) theta_sh[t] = 0ull;
  __syncthreads();

  // kTpa threads share a particle: thread `sub` takes list entries sub,
  // sub + kTpa, ...; their sums are combined by shuffles in a fixed order.
  const uint32_t sub = threadIdx.x % kTpa;
  const uint32_t i = b * kBlock + (blockIdx.x % kTpa) * kAtoms + threadIdx.x / kTpa;
  const bool real = (i - p.atom_begin) < p.n_atoms;
  const float g_pe = (float)a.obs_grad[((size_t)m * v.n_replicas + r) * 3 + 0];
  const float g_w = (float)a.obs_grad[((size_t)m * v.n_replicas + r) * 3 + 1];
  const float h_pe = 0.5f * g_pe, h_w = 0.5f * g_w;
  float gx = 0.f, gy = 0.f, gz = 0.f;
  float te[kNt], ts[kNt];
#pragma unroll
  for (int c = 0; c < kNt; ++c) te[c] = ts[c] = 0.f;
  float sa[2] = {0.f, 0.f}, sb[2] = {0.f, 0.f}, sc[2] = {0.f, 0.f}, sd[2] = {0.f, 0.f},
        sn[2] = {0.f, 0.f};
  const float4 xi = pos[i];
  const int ti = __float_as_int(xi.w);
  const AdjCoeff* row = table + ti * kNt;
  const float4 fi = a.fbar[i];
  // The list forward step m used: its snapshot, or the current (rebuilt) list.
  const uint32_t* nbr = v.nbr;
  const uint32_t* cnt = v.nbr_count;
  if (a.snap_nbr != nullptr) {
    const int src = a.list_src[r];
    const size_t s = src < 0 ? 0u : (size_t)src;
    nbr = a.snap_nbr + s * a.snap_entries;
    cnt = a.snap_cnt + s * v.n_slots;
  }
  const uint32_t n = real ? cnt[i] : 0u;  // every thread of the particle
  const uint32_t n_warp = __reduce_max_sync(kFull, n);
  const float hmin = fminf(p.half[0], fminf(p.half[1], p.half[2]));
  const float half_min_sq = hmin * hmin;
  const uint32_t* list = nbr + nbr_index(i, 0, v.nbr_stride);
  constexpr uint32_t kU = 4;
  uint32_t jn[kU];
#pragma unroll
  for (uint32_t u = 0; u < kU; ++u) {
    const uint32_t q = u * kTpa + sub;
    jn[u] = q < n ? __ldcs(list + (size_t)q * kGroup) : i;
  }
  for (uint32_t k0 = 0; k0 < n_warp; k0 += kU * kTpa) {
    uint32_t j[kU];
    float4 xj[kU], fj[kU];
#pragma unroll
    for (uint32_t u = 0; u < kU; ++u) j[u] = jn[u];
#pragma unroll
    for (uint32_t u = 0; u < kU; ++u) {
      xj[u] = __ldg(&pos[j[u]]);
      fj[u] = __ldg(&a.fbar[j[u]]);
    }
#pragma unroll
    for (uint32_t u = 0; u < kU; ++u) {
      const uint32_t q = k0 + (kU + u) * kTpa + sub;
      jn[u] = q < n ? __ldcs(list + (size_t)q * kGroup) : i;
    }
#pragma unroll
    for (uint32_t u = 0; u < kU; ++u) {
      float dx = xi.x - xj[u].x, dy = xi.y - xj[u].y, dz = xi.z - xj[u].z;
      float r2 = norm2(dx, dy, dz);
      const bool far = r2 >= half_min_sq;
      if (__any_sync(kFull, far)) {
        if (far) {
          dx = acc_delta(xi.x, xj[u].x, p.len[0], p.half[0]);
          dy = acc_delta(xi.y, xj[u].y, p.len[1], p.half[1]);
          dz = acc_delta(xi.z, xj[u].z, p.len[2], p.half[2]);
          r2 = norm2(dx, dy, dz);
        }
      }
      const bool in = (k0 + u * kTpa + sub < n) && r2 < rc2;
      const int tj = __float_as_int(xj[u].w);
      const AdjCoeff c = row[tj];
      const float rr = in ? r2 : 1.0f;
      const float inv = __fdividef(1.0f, rr);
      const float sr2 = c.sigma2 * inv;
      const float sr6 = sr2 * sr2 * sr2;
      const float sr12 = sr6 * sr6;
      const float phi = in ? c.eps24 * inv * (2.0f * sr12 - sr6) : 0.0f;
      const float psi = in ? 4.0f * c.eps24 * inv * inv * (2.0f * sr6 - 7.0f * sr12) : 0.0f;
      const float ddx = fi.x - fj[u].x, ddy = fi.y - fj[u].y, ddz = fi.z - fj[u].z;
      const float d_dot = dx * ddx + dy * ddy + dz * ddz;
      const float coef = psi * d_dot - g_pe * phi + g_w * (psi * rr + 2.0f * phi);
      gx += phi * ddx + coef * dx;
      gy += phi * ddy + coef * dy;
      gz += phi * ddz + coef * dz;
      // Parameter adjoints of this ordered pair (the pair's PE and W are
      // split half and half between its two ordered entries).
      const float fd = fi.x * dx + fi.y * dy + fi.z * dz;
      if constexpr (kNt == 2) {
        // Five per-type sums; the per-type-pair constants multiply them
        // once after the loop (see below).  With P = sr12, Q = sr6 and
        // w = F_bar_i . d + h_W r^2:  a = inv (2P - Q) w, b = P - Q,
        // c = inv (4P - Q) w, d = 2P - Q, n = 1, each masked to in-range.
        const float m = in ? 1.0f : 0.0f;
        const float tf = (float)tj, omt = 1.0f - tf;
        const float w = fd + h_w * rr;
        const float g2m = (2.0f * sr12 - sr6) * m;
        const float ea = inv * g2m * w;
        const float eb = (sr12 - sr6) * m;
        const float ec = inv * (4.0f * sr12 - sr6) * w * m;
        sa[0] += omt * ea, sa[1] += tf * ea;
        sb[0] += omt * eb, sb[1] += tf * eb;
        sc[0] += omt * ec, sc[1] += tf * ec;
        sd[0] += omt * g2m, sd[1] += tf * g2m;
        sn[0] += omt * m, sn[1] += tf * m;
      } else {
        const float uu = c.eps4 * (sr12 - sr6) - c.shift;
        const float d_eps = (phi * fd + h_pe * uu + h_w * phi * rr) * c.inv_eps;
        const float qq = 24.0f * sr12 - 6.0f * sr6;
        const float dphi = c.eps24 * inv * qq * c.inv_sig;
        const float du = c.eps4 * (12.0f * sr12 - 6.0f * sr6) * c.inv_sig - c.dshift;
        const float d_sig = dphi * fd + h_pe * du + h_w * dphi * rr;
        add_typed<kNt>(te, tj, in ? d_eps : 0.0f);
        add_typed<kNt>(ts, tj, in ? d_sig : 0.0f);
      }
    }
  }
  if constexpr (kNt == 2) {
    // d eps_t = (1/eps) [24 eps a + h_PE (4 eps b - shift n)],
    // d sigma_t = (1/sigma) [24 eps 6 c + h_PE 4 eps 6 d] - h_PE dshift n.
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const AdjCoeff ct = row[t];
      te[t] = ct.inv_eps * (ct.eps24 * sa[t] + h_pe * (ct.eps4 * sb[t] - ct.shift * sn[t]));
      ts[t] = ct.inv_sig * (6.0f * ct.eps24 * sc[t] + 6.0f * h_pe * ct.eps4 * sd[t]) -
              h_pe * ct.dshift * sn[t];
    }
  }
  if (kTpa > 1) {
#pragma unroll
    for (int o = 1; o < kTpa; o <<= 1) {
      gx += __shfl_xor_sync(kFull, gx, o);
      gy += __shfl_xor_sync(kFull, gy, o);
      gz += __shfl_xor_sync(kFull, gz, o);
    }
  }
  const bool owner = real && sub == 0u;
  double dot = 0.0;
  if (owner) {
    float4 xb = a.xbar[i];
    xb.x += gx;
    xb.y += gy;
    xb.z += gz;
    a.xbar[i] = xb;
    if (!first && finish) {
      const float4 vb = a.vbar[i];
      const float4 ub = make_float4(__fmaf_rn(p.dt, xb.x, vb.x), __fmaf_rn(p.dt, xb.y, vb.y),
                                    __fmaf_rn(p.dt, xb.z, vb.z), 0.f);
      a.ubar[i] = ub;
      const float4 vp = a.seg_vel[(size_t)(k - 1) * a.slots + i];
      dot = (double)ub.x * vp.x + (double)ub.y * vp.y + (double)ub.z * vp.z;
    }
  }
  if (!first && finish) {
    long long* dout = a.dot + ((size_t)lane_out * v.n_replicas + r) * 2;
    block_add_fixed<kBlock>(owner ? to_fixed(dot, &st->status) : Fixed{0, 0}, dout, dout + 1);
  }
  if (real) {
    for (int c = 0; c < nt; ++c) {
      const int slot = (ti * kAdjTypes + c) * 2;
      const Fixed fe = to_fixed((double)te[c], &st->status);
      const Fixed fs = to_fixed((double)ts[c], &st->status);
      atomicAdd(&theta_sh[(slot + 0) * 2 + 0], (unsigned long long)fe.whole);
      atomicAdd(&theta_sh[(slot + 0) * 2 + 1], (unsigned long long)fe.frac);
      atomicAdd(&theta_sh[(slot + 1) * 2 + 0], (unsigned long long)fs.whole);
      atomicAdd(&theta_sh[(slot + 1) * 2 + 1], (unsigned long long)fs.frac);
    }
  }
  __syncthreads();
  unsigned long long* out =
      reinterpret_cast<unsigned long long*>(a.theta) + (size_t)r * kAdjTypes * kAdjTypes * 4;
  for (int t = threadIdx.x; t < kAdjTypes * kAdjTypes * 4; t += kBlock) {
    if (theta_sh[t] != 0ull) atomicAdd(&out[t], theta_sh[t]);
  }
}

constexpr int kAdjBondedTypes = 8;  // bonded types per kind and replica the adjoint supports
constexpr int kDirs = 4;            // dual directions: F_bar, arms, parameter a, parameter b

// Minimum-image arm x_a - x_b as a dual: direction 0 carries F_bar_a -
// F_bar_b, direction 1 the arm itself (the tangent x_m - x_me of every
// member, differenced), directions 2-3 nothing.
__device__ __forceinline__ V3T<Dual<kDirs>> dual_arm(const DeviceView& v, const AdjView& a,
                                                     const ReplicaParams& p,
                                                     const float4* pos, uint32_t ta,
                                                     uint32_t tb) {
  const uint32_t sa = v.slot_of_tag[ta], sb = v.slot_of_tag[tb];
  const float4 xa = pos[sa], xb = pos[sb];
  const float4 fa = a.fbar[sa], fb = a.fbar[sb];
  const float dx = acc_delta(xa.x, xb.x, p.len[0], p.half[0]);
  const float dy = acc_delta(xa.y, xb.y, p.len[1], p.half[1]);
  const float dz = acc_delta(xa.z, xb.z, p.len[2], p.half[2]);
  V3T<Dual<kDirs>> d;
  d.x = dconst<kDirs>(dx);
  d.y = dconst<kDirs>(dy);
  d.z = dconst<kDirs>(dz);
  d.x.d[0] = fa.x - fb.x;
  d.y.d[0] = fa.y - fb.y;
  d.z.d[0] = fa.z - fb.z;
  d.x.d[1] = dx;
  d.y.d[1] = dy;
  d.z.d[1] = dz;
  return d;
}

// Step m, bonded part: x_bar += J F_bar + g_PE grad PE + g_W grad W over the
// particle's harmonic terms (forward-mode duals of the term forces), the
// k / r0 / theta0 adjoints, then (the last kernel of the step) u_bar_m and
// the sum u_bar_m . v_m-1.
__global__ void __launch_bounds__(kBlock)
k_adj_bonded(DeviceView v, AdjView a, const float4* __restrict__ pos, uint32_t m, uint32_t k,
             int first, int lane_out) {
  const uint32_t b = blockIdx.x;
  const uint32_t r = v.block_replica[b];
  const ReplicaParams& p = v.rp[r];
  ReplicaState* st = &v.rs[r];
  __shared__ unsigned long long sh[3][kAdjBondedTypes][2][2];
  for (int t = threadIdx.x; t < 3 * kAdjBondedTypes * 4; t += kBlock) {
    (&sh[0][0][0][0])[t] = 0ull;
  }
  __syncthreads();
  const uint32_t i = b * kBlock + threadIdx.x;
  const bool real = (i - p.atom_begin) < p.n_atoms;
  const float g_pe = (float)a.obs_grad[((size_t)m * v.n_replicas + r) * 3 + 0];
  const float g_w = (float)a.obs_grad[((size_t)m * v.n_replicas + r) * 3 + 1];
  float gx = 0.f, gy = 0.f, gz = 0.f;
  if (real) {
    const float4 fi = a.fbar[i];
    const uint32_t t = v.tag[i];
    const uint32_t e0 = v.term_off[t], e1 = v.term_off[t + 1];
    for (uint32_t e = e0; e < e1; ++e) {
      const uint32_t mem = v.term[e];
      const uint32_t kind = mem >> 30;
      const uint32_t role = (mem >> 28) & 3u;
      const uint32_t idx = mem & 0x0fffffffu;
      Dual<kDirs> en, vir;
      V3T<Dual<kDirs>> f;
      int kind_slot = 0, local = 0;
      if (kind == kTermBond) {
        const uint4 q = v.bonds[idx];
        const BondCoeff c = v.bond_coeff[q.z];
        Dual<kDirs> kk = dconst<kDirs>(c.k), r0 = dconst<kDirs>(c.r0);
        kk.d[2] = 1.0f;
        r0.d[3] = 1.0f;
        f = dual_bond<kDirs>(dual_arm(v, a, p, pos, q.x, q.y), kk, r0, role, en, vir);
        kind_slot = 0;
        local = (int)(q.z - p.bond_type_base);
      } else if (kind == kTermAngle) {
        const uint4 q = v.angles[idx];
        const AngleCoeff c = v.angle_coeff[q.w];
        Dual<kDirs> kk = dconst<kDirs>(c.k), th = dconst<kDirs>(c.theta0);
        kk.d[2] = 1.0f;
        th.d[3] = 1.0f;
        f = dual_angle<kDirs>(dual_arm(v, a, p, pos, q.x, q.y), dual_arm(v, a, p, pos, q.z, q.y),
                              kk, th, role, en, vir);
        kind_slot = 1;
        local = (int)(q.w - p.angle_type_base);
      } else {
        const uint4 q = v.dihedrals[idx];
        const uint32_t ty = v.dihedral_type[idx];
        const DihedralCoeff c = v.dihedral_coeff[ty];
        Dual<kDirs> kk = dconst<kDirs>(c.k);
        kk.d[2] = 1.0f;
        f = dual_dihedral<kDirs>(dual_arm(v, a, p, pos, q.x, q.y),
                                 dual_arm(v, a, p, pos, q.z, q.y),
                                 dual_arm(v, a, p, pos, q.z, q.w), kk, c.d, c.n, role, en, vir);
        kind_slot = 2;
        local = (int)(ty - p.dihedral_type_base);
      }
      // J F_bar (direction 0) + g_PE grad PE (= -F) + g_W grad W (= F + direction 1)
      gx += f.x.d[0] - g_pe * f.x.v + g_w * (f.x.v + f.x.d[1]);
      gy += f.y.d[0] - g_pe * f.y.v + g_w * (f.y.v + f.y.d[1]);
      gz += f.z.d[0] - g_pe * f.z.v + g_w * (f.z.v + f.z.d[1]);
      for (int q2 = 0; q2 < 2; ++q2) {
        const int dir = 2 + q2;
        float g = fi.x * f.x.d[dir] + fi.y * f.y.d[dir] + fi.z * f.z.d[dir];
        if (role == 0u) g += g_pe * en.d[dir] + g_w * vir.d[dir];
        if (g != 0.0f && local >= 0 && local < kAdjBondedTypes) {
          const Fixed fx = to_fixed((double)g, &st->status);
          atomicAdd(&sh[kind_slot][local][q2][0], (unsigned long long)fx.whole);
          atomicAdd(&sh[kind_slot][local][q2][1], (unsigned long long)fx.frac);
        }
      }
    }
  }
  double dot = 0.0;
  if (real) {
    float4 xb = a.xbar[i];
    xb.x += gx;
    xb.y += gy;
    xb.z += gz;
    a.xbar[i] = xb;
    if (!first) {
      const float4 vb = a.vbar[i];
      const float4 ub = make_float4(__fmaf_rn(p.dt, xb.x, vb.x), __fmaf_rn(p.dt, xb.y, vb.y),
                                    __fmaf_rn(p.dt, xb.z, vb.z), 0.f);
      a.ubar[i] = ub;
      const float4 vp = a.seg_vel[(size_t)(k - 1) * a.slots + i];
      dot = (double)ub.x * vp.x + (double)ub.y * vp.y + (double)ub.z * vp.z;
    }
  }
  if (!first) {
    long long* dout = a.dot + ((size_t)lane_out * v.n_replicas + r) * 2;
    block_add_fixed<kBlock>(real ? to_fixed(dot, &st->status) : Fixed{0, 0}, dout, dout + 1);
  }
  __syncthreads();
  for (int t = threadIdx.x; t < 3 * kAdjBondedTypes * 4; t += kBlock) {
    const unsigned long long val = (&sh[0][0][0][0])[t];
    if (val == 0ull) continue;
    const int kind_slot = t / (kAdjBondedTypes * 4);
    const int rest = t % (kAdjBondedTypes * 4);
    const int local = rest / 4, q2 = (rest / 2) % 2, word = rest % 2;
    long long* dst;
    if (kind_slot == 0) {
      dst = a.theta_bond + ((size_t)(p.bond_type_base + local) * 2 + q2) * 2 + word;
    } else if (kind_slot == 1) {
      dst = a.theta_angle + ((size_t)(p.angle_type_base + local) * 2 + q2) * 2 + word;
    } else {
      if (q2 != 0) continue;  // dihedrals have one parameter
      dst = a.theta_dihedral + (size_t)(p.dihedral_type_base + local) * 2 + word;
    }
    atomicAdd(reinterpret_cast<unsigned long long*>(dst), val);
  }
}

// Tag-order copy of a per-slot adjoint vector.
__global__ void k_adj_gather(DeviceView v, const float4* src, float* dst, uint32_t n_tags) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tags) return;
  const float4 x = src[v.slot_of_tag[t]];
  dst[3 * (size_t)t] = x.x;
  dst[3 * (size_t)t + 1] = x.y;
  dst[3 * (size_t)t + 2] = x.z;
}

void launch_check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    throw std::runtime_error(std::string("CUDA launch of ") + what + " failed: " +
                             cudaGetErrorString(e));
  }
}

}  // namespace

void Engine::set_lj(uint32_t replica, const double* eps, const double* sigma) {
  const ReplicaHost& h = rep_.at(replica);
  const int nt = h.n_types;
  std::vector<LjCoeff> table(static_cast<size_t>(nt) * nt);
  const float rc = static_cast<float>(h.lj_cutoff);
  for (int i = 0; i < nt; ++i) {
    for (int j = 0; j < nt; ++j) {
      const double e = eps[i * nt + j], s = sigma[i * nt + j];
      if (!(e >= 0.0) || !(s > 0.0) || !std::isfinite(e) || !std::isfinite(s)) {
        throw InvalidArgument("LJ epsilon must be >= 0 and sigma > 0.");
      }
      if (eps[i * nt + j] != eps[j * nt + i] || sigma[i * nt + j] != sigma[j * nt + i]) {
        throw InvalidArgument("LJ tables must be symmetric.");
      }
      LjCoeff c;
      const float sig = static_cast<float>(s);
      c.sigma2 = sig * sig;
      c.eps4 = 4.0f * static_cast<float>(e);
      c.eps24 = 6.0f * c.eps4;
      c.shift = 0.0f;
      if (h.lj_shift) {
        const float sr2 = c.sigma2 / (rc * rc);
        const float sr6 = sr2 * sr2 * sr2;
        c.shift = c.eps4 * (sr6 * sr6 - sr6);
      }
      table[static_cast<size_t>(i) * nt + j] = c;
    }
  }
  sync();
  h2d(const_cast<LjCoeff*>(v_.lj) + h.lj_offset, table.data(), table.size() * sizeof(LjCoeff),
      "LJ table upload");
  initialized_ = false;  // forces of the current state are stale
}

void Engine::adjoint_segment_storage(uint32_t K) {
  AdjointStore& A = *adj_;
  const uint32_t R = A.replicas;
  const size_t S = A.slots;
  if (A.seg_capacity >= K + 1) return;
  clear_replay_graphs();  // they record into the buffers replaced here
  A.seg_capacity = K + 1;
  // one spare entry: a list entry naming the far particle (slot S) stays in bounds
  A.seg_pos = A.alloc<float4>(static_cast<size_t>(K + 1) * S + 1);
  A.seg_vel = A.alloc<float4>(static_cast<size_t>(K + 1) * S);
  A.seg_lam = A.alloc<double>(static_cast<size_t>(K + 1) * R);
  A.seg_kin = A.alloc<double>(static_cast<size_t>(K + 1) * R);
  A.seg_flags = A.alloc<uint32_t>(static_cast<size_t>(K + 1) * R);
  A.seg_src = A.alloc<int>(static_cast<size_t>(K + 1) * R);
  A.seg_changed = A.alloc<uint32_t>(static_cast<size_t>(K + 1) * R);
}

// The replay of a segment of `steps` steps from its restored checkpoint:
// record step 0, then each step followed by its recording, captured once
// per length (the recording buffers and the step kernels are the same for
// every segment) so a segment is one graph launch instead of a few host
// calls per step.
cudaGraphExec_t Engine::replay_graph_for(uint32_t steps) {
  auto it = replay_graphs_.find(steps);
  if (it != replay_graphs_.end()) return it->second.second;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cuda_check(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal), "begin capture");
  try {
    adjoint_record(0);
    adjoint_snapshot(0, true);
    for (uint32_t k = 1; k <= steps; ++k) {
      if (use_conditional_) {
        record_step_conditional(false);
      } else {
        record_step(false);
      }
      adjoint_record(k);
      adjoint_snapshot(k, false);
    }
    cuda_check(cudaStreamEndCapture(stream_, &graph), "end capture");
    cuda_check(cudaGraphInstantiate(&exec, graph, 0), "graph instantiate");
  } catch (...) {
    cudaGraph_t discard = nullptr;
    cudaStreamEndCapture(stream_, &discard);
    if (discard) cudaGraphDestroy(discard);
    if (graph) cudaGraphDestroy(graph);
    throw;
  }
  replay_graphs_[steps] = std::make_pair(graph, exec);
  return exec;
}

void Engine::adjoint_record(uint32_t k) {
  AdjointStore& A = *adj_;
  const size_t S = A.slots;
  cuda_check(cudaMemcpyAsync(A.seg_pos + k * S, v_.pos, S * sizeof(float4),
                             cudaMemcpyDeviceToDevice, stream_), "adjoint record");
  cuda_check(cudaMemcpyAsync(A.seg_vel + k * S, v_.vel, S * sizeof(float4),
                             cudaMemcpyDeviceToDevice, stream_), "adjoint record");
  k_adj_record<<<(A.replicas + 127) / 128, 128, 0, stream_>>>(v_, A.seg_lam, A.seg_kin,
                                                               A.seg_flags, k);
  launch_check("adjoint record");
}

// Snapshot k of the list (see k_adj_snapshot); nothing when the backward
// pass rebuilds its lists instead.
void Engine::adjoint_snapshot(uint32_t k, bool all) {
  AdjointStore& A = *adj_;
  if (!A.snap_on) return;
  k_adj_snapshot<<<v_.n_blocks, 256, 0, stream_>>>(v_, A.snap_nbr, A.snap_cnt, k, all ? 1 : 0);
  launch_check("adjoint list snapshot");
}

// Puts the particle state of checkpoint c back, with the neighbour list the
// forward run had at that point (rebuilt from its build positions) and the
// forces of that state.
void Engine::adjoint_restore(uint32_t c) {
  AdjointStore& A = *adj_;
  const size_t S = A.slots;
  auto d2d = [&](void* dst, const void* src, size_t bytes) {
    cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream_),
               "adjoint restore");
  };
  d2d(v_.pos, A.ck_ref_pos + c * S, S * sizeof(float4));
  d2d(v_.img, A.ck_ref_img + c * S, S * sizeof(int4));
  k_adj_mark_all<<<(A.replicas + 127) / 128, 128, 0, stream_>>>(v_);
  launch_check("adjoint mark");
  launch_rebuild(launch_, false);
  d2d(v_.pos, A.ck_pos + c * S, S * sizeof(float4));
  d2d(v_.vel, A.ck_vel + c * S, S * sizeof(float4));
  d2d(v_.img, A.ck_img + c * S, S * sizeof(int4));
  d2d(v_.ref_pos, A.ck_ref_pos + c * S, S * sizeof(float4));
  d2d(v_.ref_img, A.ck_ref_img + c * S, S * sizeof(int4));
  k_adj_cross<<<(static_cast<uint32_t>(S) + kBlock - 1) / kBlock, kBlock, 0, stream_>>>(v_);
  launch_check("adjoint crossings");
  cuda_check(cudaMemcpyAsync(v_.rs, A.ck_state.data() + static_cast<size_t>(c) * A.replicas,
                             A.replicas * sizeof(ReplicaState), cudaMemcpyHostToDevice, stream_),
             "adjoint restore");
  // The next step's pre-kick reads the forces of this state: recompute them
  // on the restored list (every schedule sums in the same order, so these
  // are the forward run's bits).
  launch_forces(launch_, false, false, false);
  sync();
}

void Engine::adjoint_forward(uint64_t steps, uint64_t record_from, uint32_t every, double* obs) {
  TraceRange trace("beads.adjoint_forward");
  if (steps == 0) throw InvalidArgument("adjoint runs need at least one step.");
  if (record_from > steps) throw InvalidArgument("record_from must not exceed steps.");
  for (const auto& h : rep_) {
    if (h.n_bond_types > 8 || h.n_angle_types > 8 || h.n_dihedral_types > 8) {
      throw InvalidArgument("the adjoint supports up to 8 bonded types of each kind per replica.");
    }
  }
  int max_types = 0;
  for (const auto& h : rep_) max_types = std::max(max_types, h.n_types);
  if (max_types > kAdjTypes) throw InvalidArgument("the adjoint supports up to 4 particle types.");
  // The adjoint pair kernel reads slot rows of slot entries: leave the staged
  // list layout (same forward bits, the list is rebuilt in slot layout).
  set_list_staged(false);

  if (!adj_) adj_ = std::make_unique<AdjointStore>();
  AdjointStore& A = *adj_;
  A.stream = stream_;
  const uint32_t R = n_replicas();
  const size_t S = v_.n_slots;
  // every == 0: keep every step's state from this forward pass (one segment,
  // no replay in the backward pass) -- the trade of memory for compute that
  // 180 GB of HBM usually affords: 32 bytes per slot and step.
  A.store_all = every == 0;
  if (A.store_all) {
    if (steps > 0xFFFFFFF0ull) throw InvalidArgument("too many steps to store.");
    every = static_cast<uint32_t>(steps);
  }
  A.steps = steps;
  A.record_from = record_from;
  A.every = every;
  A.segments = static_cast<uint32_t>((steps + every - 1) / every);
  A.slots = static_cast<uint32_t>(S);
  A.replicas = R;
  A.max_types = max_types;
  if (A.ck_capacity < A.segments + 1ull) {
    A.ck_capacity = A.segments + 1ull;
    A.ck_pos = A.alloc<float4>(A.ck_capacity * S);
    A.ck_vel = A.alloc<float4>(A.ck_capacity * S);
    A.ck_img = A.alloc<int4>(A.ck_capacity * S);
    A.ck_ref_pos = A.alloc<float4>(A.ck_capacity * S);
    A.ck_ref_img = A.alloc<int4>(A.ck_capacity * S);
  }
  A.ck_state.assign(static_cast<size_t>(A.segments + 1) * R, ReplicaState{});
  A.forward_done = false;

  // Slots must not move during an adjoint run: switch off the periodic
  // reorder on the device (restored at the end of the backward pass).
  set_sort_enabled(false);

  auto save = [&](uint32_t c) {
    auto d2d = [&](void* dst, const void* src, size_t bytes) {
      cuda_check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream_),
                 "checkpoint");
    };
    d2d(A.ck_pos + c * S, v_.pos, S * sizeof(float4));
    d2d(A.ck_vel + c * S, v_.vel, S * sizeof(float4));
    d2d(A.ck_img + c * S, v_.img, S * sizeof(int4));
    d2d(A.ck_ref_pos + c * S, v_.ref_pos, S * sizeof(float4));
    d2d(A.ck_ref_img + c * S, v_.ref_img, S * sizeof(int4));
    sync();
    d2h(A.ck_state.data() + static_cast<size_t>(c) * R, v_.rs, R * sizeof(ReplicaState), "checkpoint");
  };
  std::vector<beads_observables> o;
  auto put_obs = [&](uint64_t n) {
    observables(o);
    for (uint32_t r = 0; r < R; ++r) {
      double* row = obs + ((n - record_from) * R + r) * 3;
      row[0] = o[r].pe;
      row[1] = o[r].virial;
      row[2] = o[r].ke;
    }
  };

  eval();
  if (!tuned_ && !tuning_fixed_) autotune();
  save(0);
  if (record_from == 0) put_obs(0);
  if (A.store_all) {
    adjoint_segment_storage(every);
    adjoint_record(0);
  }
  uint64_t n = 0;
  while (n < steps) {
    const uint64_t next_ck = (n / every + 1) * every;
    if (A.store_all) {
      run(1, n + 1 >= record_from ? 1 : 0);
      n += 1;
      adjoint_record(static_cast<uint32_t>(n));
      if (n >= record_from) put_obs(n);
    } else if (n + 1 >= record_from) {
      run(1, 1);
      n += 1;
      put_obs(n);
    } else {
      const uint64_t upto = std::min({next_ck, record_from - 1, steps});
      run(upto - n, 0);
      n = upto;
    }
    if (n % every == 0 && n < steps) save(static_cast<uint32_t>(n / every));
  }
  save(A.segments);  // the final state
  A.forward_done = true;
}

void Engine::adjoint_backward(const double* obs_grad, double* grad_eps, double* grad_sigma,
                              float* grad_pos, float* grad_vel) {
  TraceRange trace("beads.adjoint_backward");
  if (!adj_ || !adj_->forward_done) throw InvalidArgument("adjoint_backward needs a forward run.");
  AdjointStore& A = *adj_;
  const uint32_t R = A.replicas;
  const size_t S = A.slots;
  const uint64_t T = A.steps;
  const uint32_t K = A.every;

  adjoint_segment_storage(K);
  // List snapshots for the reverse sweep when the device holds K + 1 of them
  // with room to spare (a replayed segment records them; storing every step
  // in the forward pass has no replay and rebuilds instead).
  {
    const uint64_t want = static_cast<uint64_t>(K) + 1u;
    const uint64_t bytes = want * S * (static_cast<uint64_t>(v_.nbr_stride) + 1u) * 4u;
    bool on = false;
    if (!A.store_all) {
      if (A.snap_capacity >= want) {
        on = true;
      } else {
        size_t free_b = 0, total_b = 0;
        cuda_check(cudaMemGetInfo(&free_b, &total_b), "memory info");
        if (bytes <= free_b / 2) {
          clear_replay_graphs();  // they copy into the buffers replaced here
          A.snap_nbr = A.alloc<uint32_t>(want * S * v_.nbr_stride);
          A.snap_cnt = A.alloc<uint32_t>(want * S);
          A.snap_capacity = static_cast<uint32_t>(want);
          on = true;
        }
      }
    }
    if (on != A.snap_on) clear_replay_graphs();  // they hold (or lack) the snapshot copies
    A.snap_on = on;
  }
  if (!A.xbar) {
    A.xbar = A.alloc<float4>(S);
    A.vbar = A.alloc<float4>(S);
    A.fbar = A.alloc<float4>(S + 1);  // + the far particle's (zero) entry
    A.ubar = A.alloc<float4>(S);
    A.theta = A.alloc<long long>(static_cast<size_t>(R) * kAdjTypes * kAdjTypes * 4);
    A.tag_xfer = A.alloc<float>(3 * n_tags_);
    A.shift_on = A.alloc<int>(R);
    A.dot = A.alloc<long long>(static_cast<size_t>(R) * 4);
    A.theta_bond = A.alloc<long long>(std::max<size_t>(1, total_bond_types_) * 4);
    A.theta_angle = A.alloc<long long>(std::max<size_t>(1, total_angle_types_) * 4);
    A.theta_dihedral = A.alloc<long long>(std::max<size_t>(1, total_dihedral_types_) * 2);
  }
  if (A.obs_capacity < (T + 1) * R * 3) {
    A.obs_capacity = (T + 1) * R * 3;
    A.obs_grad = A.alloc<double>(A.obs_capacity);
  }
  int* d_shift = A.shift_on;
  {
    std::vector<double> g((T + 1) * R * 3, 0.0);
    std::copy(obs_grad, obs_grad + (T + 1 - A.record_from) * R * 3,
              g.begin() + A.record_from * R * 3);
    h2d(A.obs_grad, g.data(), g.size() * sizeof(double), "adjoint upload");
    std::vector<int> sh(R);
    for (uint32_t r = 0; r < R; ++r) sh[r] = rep_[r].lj_shift ? 1 : 0;
    h2d(d_shift, sh.data(), R * sizeof(int), "adjoint upload");
  }
  sync();
  cuda_check(cudaMemsetAsync(A.xbar, 0, S * sizeof(float4), stream_), "memset");
  cuda_check(cudaMemsetAsync(A.ubar, 0, S * sizeof(float4), stream_), "memset");
  cuda_check(cudaMemsetAsync(A.vbar, 0, S * sizeof(float4), stream_), "memset");
  cuda_check(cudaMemsetAsync(A.theta, 0, static_cast<size_t>(R) * kAdjTypes * kAdjTypes * 4 * 8,
             stream_),
             "memset");
  cuda_check(cudaMemsetAsync(A.dot, 0, static_cast<size_t>(R) * 4 * sizeof(long long), stream_),
             "memset");
  cuda_check(cudaMemsetAsync(A.theta_bond, 0, std::max<size_t>(1, total_bond_types_) * 4 * 8,
             stream_), "memset");
  cuda_check(cudaMemsetAsync(A.theta_angle, 0, std::max<size_t>(1, total_angle_types_) * 4 * 8, stream_),
             "memset");
  cuda_check(cudaMemsetAsync(A.theta_dihedral, 0, std::max<size_t>(1,
             total_dihedral_types_) * 2 * 8, stream_),
             "memset");

  AdjView av{};
  av.seg_pos = A.seg_pos;
  av.seg_vel = A.seg_vel;
  av.seg_lam = A.seg_lam;
  av.seg_kin = A.seg_kin;
  av.xbar = A.xbar;
  av.vbar = A.vbar;
  av.fbar = A.fbar;
  av.ubar = A.ubar;
  av.obs_grad = A.obs_grad;
  av.theta = A.theta;
  av.ck_ref_pos = A.ck_ref_pos;
  av.list_src = nullptr;
  av.snap_nbr = A.snap_on ? A.snap_nbr : nullptr;
  av.snap_cnt = A.snap_on ? A.snap_cnt : nullptr;
  av.snap_entries = static_cast<uint64_t>(S) * v_.nbr_stride;
  av.shift_on = d_shift;
  av.dot = A.dot;
  av.theta_bond = A.theta_bond;
  av.theta_angle = A.theta_angle;
  av.theta_dihedral = A.theta_dihedral;
  av.slots = A.slots;
  av.replicas = R;

  std::vector<uint32_t> flags;
  std::vector<int> current(R), src_all;
  std::vector<uint32_t> chg_all;
  std::vector<char> any_k;
  for (int s = static_cast<int>(A.segments) - 1; s >= 0; --s) {
    const uint64_t a = static_cast<uint64_t>(s) * K;
    const uint64_t b = std::min<uint64_t>(a + K, T);
    // Replay the segment, recording every step (kept from the forward pass
    // when it stored every step).
    if (!A.store_all) {
      adjoint_restore(static_cast<uint32_t>(s));
      if (use_graphs_) {
        cuda_check(cudaGraphLaunch(replay_graph_for(static_cast<uint32_t>(b - a)), stream_),
                   "replay launch");
      } else {
        adjoint_record(0);
        adjoint_snapshot(0, true);
        for (uint64_t k = 1; k <= b - a; ++k) {
          launch_chunk(1, false);
          adjoint_record(static_cast<uint32_t>(k));
          adjoint_snapshot(static_cast<uint32_t>(k), false);
        }
      }
    }
    sync();
    flags.resize(static_cast<size_t>(b - a + 1) * R);
    d2h(flags.data(), A.seg_flags, flags.size() * sizeof(uint32_t), "flags");
    // The list each forward step m used: built at the replica's last rebuild
    // at or before m inside this segment, else the checkpoint's.  Walking
    // backwards, a replica's list is rebuilt when that source changes; the
    // sources and change flags of the whole segment go to the device at once.
    std::fill(current.begin(), current.end(), -2);  // list state unknown
    const uint64_t m_lo = (s == 0) ? 0 : a + 1;
    const size_t nk = static_cast<size_t>(b - a + 1);
    src_all.assign(nk * R, -1);
    chg_all.assign(nk * R, 0u);
    any_k.assign(nk, 0);
    for (uint64_t m = b + 1; m-- > m_lo;) {
      const uint32_t k = static_cast<uint32_t>(m - a);
      for (uint32_t r = 0; r < R; ++r) {
        int src = -1;
        for (uint32_t q = k; q >= 1; --q) {
          if (flags[static_cast<size_t>(q) * R + r]) {
            src = static_cast<int>(q);
            break;
          }
        }
        src_all[k * R + r] = src;
        if (src != current[r]) {
          chg_all[k * R + r] = 1u;
          any_k[k] = 1;
          current[r] = src;
        }
      }
    }
    h2d(A.seg_src, src_all.data(), nk * R * sizeof(int), "adjoint list sources");
    h2d(A.seg_changed, chg_all.data(), nk * R * sizeof(uint32_t), "adjoint list sources");
    for (uint64_t m = b + 1; m-- > m_lo;) {
      const uint32_t k = static_cast<uint32_t>(m - a);
      AdjView lv = av;
      lv.list_src = A.seg_src + static_cast<size_t>(k) * R;
      if (any_k[k] && !A.snap_on) {
        k_adj_list_positions<<<v_.n_blocks, kBlock, 0, stream_>>>(
            v_, lv, static_cast<uint32_t>(s), A.seg_changed + static_cast<size_t>(k) * R);
        launch_check("adjoint list positions");
        launch_rebuild(launch_, false);
      }
      const int first = (m == 0) ? 1 : 0;
      const int last = (m == T) ? 1 : 0;
      const int lane_in = static_cast<int>((m + 1) & 1u);
      const int lane_out = static_cast<int>(m & 1u);
      k_adj_prepare<<<v_.n_blocks, kBlock, 0, stream_>>>(v_, av, static_cast<uint32_t>(m), k,
                                                        first, last, lane_in);
      launch_check("adjoint prepare");
      const float4* pos_m = A.seg_pos + static_cast<size_t>(k) * S;
      const int bonded = v_.has_bonded ? 1 : 0;
      // One thread per particle: on the 64 x 8192 fit the reverse sweep ran
      // 16% faster than with two threads per particle and 40% faster than
      // with four (the kernel is latency-bound at 80 registers).
      const dim3 grid(v_.n_blocks);
      const uint32_t mm = static_cast<uint32_t>(m);
      if (A.max_types <= 2) {
        k_adj_lj<2, 1><<<grid, kBlock, 0, stream_>>>(v_, lv, pos_m, mm, k, first, lane_out,
                                                     !bonded);
      } else {
        k_adj_lj<4, 1><<<grid, kBlock, 0, stream_>>>(v_, lv, pos_m, mm, k, first, lane_out,
                                                     !bonded);
      }
      launch_check("adjoint pair");
      if (bonded) {
        k_adj_bonded<<<v_.n_blocks, kBlock, 0, stream_>>>(v_, av, pos_m, static_cast<uint32_t>(m),
                                                         k, first, lane_out);
        launch_check("adjoint bonded");
      }
    }
    sync();
  }

  // Outputs.
  const uint32_t tb = static_cast<uint32_t>((n_tags_ + 255) / 256);
  k_adj_gather<<<tb, 256, 0, stream_>>>(v_, A.xbar, A.tag_xfer, static_cast<uint32_t>(n_tags_));
  launch_check("adjoint gather");
  cuda_check(cudaMemcpyAsync(grad_pos, A.tag_xfer, 3 * n_tags_ * sizeof(float),
                             cudaMemcpyDeviceToHost, stream_), "adjoint download");
  sync();
  k_adj_gather<<<tb, 256, 0, stream_>>>(v_, A.vbar, A.tag_xfer, static_cast<uint32_t>(n_tags_));
  launch_check("adjoint gather");
  cuda_check(cudaMemcpyAsync(grad_vel, A.tag_xfer, 3 * n_tags_ * sizeof(float),
                             cudaMemcpyDeviceToHost, stream_), "adjoint download");
  std::vector<long long> th(static_cast<size_t>(R) * kAdjTypes * kAdjTypes * 4);
  sync();
  d2h(th.data(), A.theta, th.size() * sizeof(long long), "adjoint download");
  size_t out = 0;
  for (uint32_t r = 0; r < R; ++r) {
    const int nt = rep_[r].n_types;
    for (int i = 0; i < nt; ++i) {
      for (int j = 0; j < nt; ++j) {
        const size_t base = ((static_cast<size_t>(r) * kAdjTypes + i) * kAdjTypes + j) * 4;
        grad_eps[out] = static_cast<double>(th[base + 0]) +
                        static_cast<double>(th[base + 1]) / kFixFrac;
        grad_sigma[out] = static_cast<double>(th[base + 2]) +
                          static_cast<double>(th[base + 3]) / kFixFrac;
        ++out;
      }
    }
  }
  // Back to the end-of-forward state, list included.
  adjoint_restore(A.segments);
  set_sort_enabled(true);
  check_status();
}

void Engine::adjoint_bonded_grads(double* grad_bond, double* grad_angle, double* grad_dihedral) {
  if (!adj_ || !adj_->theta_bond) throw InvalidArgument("no adjoint_backward has run.");
  AdjointStore& A = *adj_;
  sync();
  auto read = [&](const long long* src, size_t n_pairs, std::vector<double>& out) {
    std::vector<long long> raw(2 * std::max<size_t>(1, n_pairs));
    d2h(raw.data(), src, raw.size() * sizeof(long long), "adjoint download");
    out.resize(n_pairs);
    for (size_t q = 0; q < n_pairs; ++q) {
      out[q] = static_cast<double>(raw[2 * q]) + static_cast<double>(raw[2 * q + 1]) / kFixFrac;
    }
  };
  std::vector<double> b, an, d;
  read(A.theta_bond, 2ull * total_bond_types_, b);
  read(A.theta_angle, 2ull * total_angle_types_, an);
  read(A.theta_dihedral, total_dihedral_types_, d);
  constexpr double kPerDegree = 3.14159265358979323846 / 180.0;
  if (grad_bond) std::copy(b.begin(), b.end(), grad_bond);
  if (grad_angle) {
    for (size_t t = 0; t < total_angle_types_; ++t) {
      grad_angle[2 * t] = an[2 * t];
      grad_angle[2 * t + 1] = an[2 * t + 1] * kPerDegree;
    }
  }
  if (grad_dihedral) std::copy(d.begin(), d.end(), grad_dihedral);
}

void Engine::set_bonded(uint32_t replica, const double* bond_k, const double* bond_r0,
                        const double* angle_k, const double* angle_theta0_deg,
                        const double* dihedral_k) {
  const ReplicaHost& h = rep_.at(replica);
  sync();
  if (h.n_bond_types > 0 && (bond_k || bond_r0)) {
    std::vector<BondCoeff> c(h.n_bond_types);
    d2h(c.data(), v_.bond_coeff + h.bond_type_base, c.size() * sizeof(BondCoeff), "bonded");
    for (int t = 0; t < h.n_bond_types; ++t) {
      if (bond_k) c[t].k = static_cast<float>(bond_k[t]);
      if (bond_r0) c[t].r0 = static_cast<float>(bond_r0[t]);
    }
    h2d(const_cast<BondCoeff*>(v_.bond_coeff) + h.bond_type_base, c.data(),
        c.size() * sizeof(BondCoeff), "bonded");
  }
  if (h.n_angle_types > 0 && (angle_k || angle_theta0_deg)) {
    std::vector<AngleCoeff> c(h.n_angle_types);
    d2h(c.data(), v_.angle_coeff + h.angle_type_base, c.size() * sizeof(AngleCoeff), "bonded");
    for (int t = 0; t < h.n_angle_types; ++t) {
      if (angle_k) c[t].k = static_cast<float>(angle_k[t]);
      if (angle_theta0_deg) {
        c[t].theta0 = static_cast<float>(angle_theta0_deg[t]) * 3.14159265358979323846f / 180.0f;
      }
    }
    h2d(const_cast<AngleCoeff*>(v_.angle_coeff) + h.angle_type_base, c.data(),
        c.size() * sizeof(AngleCoeff), "bonded");
  }
  if (h.n_dihedral_types > 0 && dihedral_k) {
    std::vector<DihedralCoeff> c(h.n_dihedral_types);
    d2h(c.data(), v_.dihedral_coeff + h.dihedral_type_base, c.size() * sizeof(DihedralCoeff), "bonded");
    for (int t = 0; t < h.n_dihedral_types; ++t) c[t].k = static_cast<float>(dihedral_k[t]);
    h2d(const_cast<DihedralCoeff*>(v_.dihedral_coeff) + h.dihedral_type_base, c.data(),
        c.size() * sizeof(DihedralCoeff), "bonded");
  }
  initialized_ = false;
}

}  // namespace bb
