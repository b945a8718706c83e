// models.cuh — per-neuron model arithmetic for the sm_100a kernels.
//
// Each function advances one neuron by one step and returns whether it
// spiked.  The arithmetic reproduces the reference model operation by
// operation in FP32: the library is compiled with -fmad=false so no a*b+c is
// contracted (Rust never contracts), and __fmaf_rn appears exactly where the
// reference calls mul_add.  Division and square root are IEEE (no fast-math).
// Paths are relative to crates/SiMuse/crates/ (P/ = pillars/src/).
#pragma once
#include <cstdint>

namespace sg {

enum Model : int { kLIF = 1, kIZH = 2, kGPEA = 3, kHH = 4 };

__host__ __device__ constexpr int n_params(int m) {
  return m == kLIF ? 6 : m == kIZH ? 7 : m == kGPEA ? 14 : m == kHH ? 10 : -1;
}
__host__ __device__ constexpr int n_state(int m) {
  return m == kLIF ? 2 : m == kIZH ? 3 : m == kGPEA ? 9 : m == kHH ? 4 : -1;
}
// P/core/exec/population.rs:69-86 (CLAMP_I_SYN); GPEA is #[no_clamp]
// (P/zoo/neurons/gpea.rs:210) and the HH conductance model has no clamp.
__host__ __device__ constexpr bool clamps(int m) { return m == kLIF || m == kIZH; }

// Natural log for the GPEA calcium Nernst potential, correctly rounded to
// FP32 and compiled identically for the host and the device (so host-built
// constants, the kernels and a host restatement agree bit for bit).  Method:
// x = m * 2^k with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
// s = (m - 1)/(m + 1), by the series 2s (1 + s^2/3 + s^4/5 + ... + s^24/25)
// (Abramowitz & Stegun 4.1.27) evaluated in FP64 (|s| <= 0.1716, so the
// truncation error is below 2^-70), plus k ln 2 with ln 2 split in a short
// high part and a low correction, rounded once to FP32.  Every FP64 step is
// an IEEE add, multiply or divide (no contraction), so the result is the same
// on any IEEE machine.  Checked correctly rounded over every float in
// [1e-12, 1e6].
__host__ __device__ inline float sg_logf(float x) {
#ifdef __CUDA_ARCH__
  uint32_t b = __float_as_uint(x);
#else
  uint32_t b;
  __builtin_memcpy(&b, &x, 4);
#endif
  if (!(x > 0.0f)) return x == 0.0f ? -__builtin_huge_valf() : __builtin_nanf("");
  if (b >= 0x7f800000u) return x;  // +inf
  int k = 0;
  if (b < 0x00800000u) {  // subnormal: scale into the normal range
    x = x * 16777216.0f;
#ifdef __CUDA_ARCH__
    b = __float_as_uint(x);
#else
    __builtin_memcpy(&b, &x, 4);
#endif
    k = -24;
  }
  k += (int)(b >> 23) - 127;
  const uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
  float mf;
#ifdef __CUDA_ARCH__
  mf = __uint_as_float(mb);
#else
  __builtin_memcpy(&mf, &mb, 4);
#endif
  double m = (double)mf;
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    k += 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 25.0;
  p = p * z + 1.0 / 23.0;
  p = p * z + 1.0 / 21.0;
  p = p * z + 1.0 / 19.0;
  p = p * z + 1.0 / 17.0;
  p = p * z + 1.0 / 15.0;
  p = p * z + 1.0 / 13.0;
  p = p * z + 1.0 / 11.0;
  p = p * z + 1.0 / 9.0;
  p = p * z + 1.0 / 7.0;
  p = p * z + 1.0 / 5.0;
  p = p * z + 1.0 / 3.0;
  p = p * z + 1.0;
  const double lm = (2.0 * s) * p;
  const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10;
  return (float)((double)k * ln2_hi + ((double)k * ln2_lo + lm));
}

// P/math/fast_exp.rs:23-68 — the project's polynomial exp (fused flavour).
__device__ __forceinline__ float fast_exp(float x) {
  const float log2e = 1.44269504088896340736f;
  float t = x * log2e;
  float tf = floorf(t);
  int n = (int)tf;  // cvt.rzi saturates; NaN -> 0
  float f = t - (float)n;
  float poly = __fmaf_rn(0.0001540353f, f, 0.001333356f);
  poly = __fmaf_rn(poly, f, 0.009618129f);
  poly = __fmaf_rn(poly, f, 0.05550411f);
  poly = __fmaf_rn(poly, f, 0.2402265f);
  poly = __fmaf_rn(poly, f, 0.693147180559945309417f);
  poly = __fmaf_rn(poly, f, 1.0f);
  if (n < -126) return 0.0f;
  if (n > 127) return __int_as_float(0x7f800000);
  return __int_as_float((n + 127) << 23) * poly;
}

// Receptor kinetics of SynapticBrain (pillars-connectome/src/synaptic.rs):
// receptor codes 0 AMPA, 1 NMDA, 2 GABA_A, 3 GABA_B, 4 nAChR, 5 GluCl,
// 6 mAChR (any other code is AMPA, P/kernels/synapse/receptor.rs:103-115),
// decay time constants (ms) and reversal potentials (mV) of :71-100.
constexpr int kReceptors = 7;
__host__ __device__ constexpr float rec_tau(int r) {
  return r == 0 ? 2.0f : r == 1 ? 50.0f : r == 2 ? 10.0f : r == 3 ? 200.0f : r == 4 ? 3.0f : r == 5 ? 5.0f : 150.0f;
}
__host__ __device__ constexpr float rec_erev(int r) {
  return r == 2 ? -65.0f : (r == 3 || r == 6) ? -90.0f : r == 5 ? -70.0f : 0.0f;
}

// P/kernels/synapse/receptor.rs:126-131 nmda_mg_block(v) =
// 1 / (1 + 0.33 fast_exp(clamp(-0.06 v, -10, 10))); the SIMD form of :135-143
// gives the same bits.  Correctly rounded division.
__device__ __forceinline__ float nmda_mg_block(float v) {
  float a = -0.06f * v;
  a = a < -10.0f ? -10.0f : a;
  a = a > 10.0f ? 10.0f : a;
  return __fdiv_rn(1.0f, 1.0f + 0.33f * fast_exp(a));
}

// Exponential for the HH rates: Cody-Waite reduction by ln 2 (split in a
// short high part and a low correction), degree-7 Taylor polynomial of e^r
// on |r| <= ln2/2, and 2^k applied as two exact power-of-two factors.  The
// same definition runs on the host, so device and host agree bit for bit.
__device__ __forceinline__ float sg_expf(float x) {
  x = fminf(fmaxf(x, -87.0f), 88.0f);
  const float k = rintf(x * 1.44269504088896340736f);
  float r = __fmaf_rn(-k, 0.693145751953125f, x);
  r = __fmaf_rn(-k, 1.428606820309417232e-6f, r);
  float p = 1.0f / 5040.0f;
  p = __fmaf_rn(p, r, 1.0f / 720.0f);
  p = __fmaf_rn(p, r, 1.0f / 120.0f);
  p = __fmaf_rn(p, r, 1.0f / 24.0f);
  p = __fmaf_rn(p, r, 1.0f / 6.0f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  const int ki = (int)k;
  const int k1 = ki / 2, k2 = ki - k1;
  return (p * __int_as_float((k1 + 127) << 23)) * __int_as_float((k2 + 127) << 23);
}

// One neuron held in registers: state loaded/stored by the caller (128-bit
// accesses of 4 neighbours), parameters uniform or loaded per neuron.
template <int NS, int NP> struct RegNeuron {
  mutable float s[NS];
  float p[NP];
  __device__ __forceinline__ float &st(int c) const { return s[c]; }
  __device__ __forceinline__ float pr(int c) const { return p[c]; }
};

// One neuron's view of its population's SoA arrays.  Parameter columns that
// hold one value for the whole population are passed as kernel arguments
// (bit c of umask) instead of being read per neuron.
struct Soa {
  float *s;            // state [col][cap]
  const float *p;      // params [col][cap]
  uint32_t cap, i;
  uint32_t umask;
  const float *uval;
  __device__ __forceinline__ float &st(int c) const { return s[(size_t)c * cap + i]; }
  __device__ __forceinline__ float pr(int c) const {
    return ((umask >> c) & 1u) ? uval[c] : __ldg(&p[(size_t)c * cap + i]);
  }
};

// P/zoo/neurons/lif.rs:47-78
template <class A> __device__ __forceinline__ bool lif_step(const A &c, float i_syn, float dt) {
  float v = c.st(0), refr = c.st(1);
  const float inv_tau = c.pr(1), v_rest = c.pr(2), v_th = c.pr(3), v_reset = c.pr(4),
              tau_ref = c.pr(5);
  const bool is_refr = refr > 0.0f;
  const float dv = ((v_rest - v) + i_syn) * inv_tau * dt;
  const float v_new = v + dv;
  const bool spike = is_refr ? false : (v_new >= v_th);
  const float v_final = spike ? v_reset : v_new;
  c.st(0) = is_refr ? v : v_final;
  const float refr_set = spike ? tau_ref : (refr - dt);
  c.st(1) = fmaxf(refr_set, 0.0f);
  return spike;
}

// P/zoo/neurons/izhikevich.rs:71-125 (two 0.5*dt Euler half-steps on v,
// du from the pre-integration v, refractory freezes v at c)
template <class A> __device__ __forceinline__ bool izh_step(const A &c, float i_syn, float dt) {
  const float vs = c.st(0), u = c.st(1), refr = c.st(2);
  const float a = c.pr(1), b = c.pr(2), cc = c.pr(3), d = c.pr(4), tau_ref = c.pr(5),
              v_th = c.pr(6);
  const bool is_refr = refr > 0.0f;
  const float v = is_refr ? cc : vs;
  const float half_dt = dt * 0.5f;
  const float v_poly1 = v * (0.04f * v + 5.0f);
  const float dv1 = (v_poly1 + 140.0f - u + i_syn) * half_dt;
  const float v_mid = v + dv1;
  const float v_poly2 = v_mid * (0.04f * v_mid + 5.0f);
  const float dv2 = (v_poly2 + 140.0f - u + i_syn) * half_dt;
  const float dv_total = is_refr ? 0.0f : dv1 + dv2;
  const float v_new = v + dv_total;
  const float du = a * (b * v - u) * dt;
  const float u_new = is_refr ? u : u + du;
  const bool spike = v_new >= v_th;
  c.st(0) = spike ? cc : v_new;
  c.st(1) = spike ? u_new + d : u_new;
  const float refr_set = spike ? tau_ref : (refr - dt);
  c.st(2) = fmaxf(refr_set, 0.0f);
  return spike;
}

// ---- GPEA: P/zoo/neurons/gpea.rs:53-123 constants, 129-179 helpers, 266-360 step
namespace gp {
constexpr float NA_TH_M = -38.0f, NA_TH_H = -45.5f, NA_K_M = -7.0f, NA_K_H = 6.4f;
constexpr float NA_TAU_M0 = 0.001f, NA_TAU_M1 = 0.1f, NA_THT_M = -53.0f, NA_SIG_M = -0.7f;
constexpr float NA_TAU_H0 = 0.0f, NA_TAU_H1 = 4.5f, NA_THT_H1 = -50.0f, NA_SIG_H1 = -15.0f;
constexpr float NA_THT_H2 = -50.0f, NA_SIG_H2 = 16.0f;
constexpr float K_TH_N = -42.0f, K_K_N = -14.0f, K_TAU_N0 = 0.0f, K_TAU_N1 = 2.4f;
constexpr float K_THT_N1 = -40.0f, K_SIG_N1 = -40.0f, K_THT_N2 = -40.0f, K_SIG_N2 = 50.0f;
constexpr float CAT_TH_P = -56.0f, CAT_TH_Q = -85.0f, CAT_K_P = -6.7f, CAT_K_Q = 5.8f;
constexpr float CAT_TAU_P0 = 5.0f, CAT_TAU_P1 = 0.33f, CAT_TAU_Q0 = 0.0f, CAT_TAU_Q1 = 400.0f;
constexpr float CAT_THT_P1 = -27.0f, CAT_SIG_P1 = -10.0f, CAT_THT_P2 = -102.0f, CAT_SIG_P2 = 15.0f;
constexpr float CAT_THT_Q1 = -50.0f, CAT_SIG_Q1 = -15.0f, CAT_THT_Q2 = -50.0f, CAT_SIG_Q2 = 16.0f;
constexpr float AHP_TH_R = 0.17e-3f, AHP_K_R = -0.08e-3f, AHP_TAU_R = 2.0f;
constexpr float CA_FARADAY = 96485.0f, CA_CAO = 2.0f, GAS_R = 8.31441f;
}  // namespace gp

__device__ __forceinline__ float gp_sigmoid(float x, float th, float inv_k) {
  return 1.0f / (1.0f + fast_exp((x - th) * inv_k));
}
__device__ __forceinline__ float gp_exp_euler(float x, float x_inf, float tau, float dt) {
  const float decay = fast_exp(-dt / tau);
  return __fmaf_rn(decay, x - x_inf, x_inf);
}
__device__ __forceinline__ float gp_tau2(float v, float t0, float t1, float th1, float m1,
                                         float th2, float m2) {
  const float e1 = fast_exp((v - th1) * m1);
  const float e2 = fast_exp((-(v - th2)) * m2);
  return t0 + t1 / (e1 + e2);
}

// ln(NAI/NAO) and ln(KO/KI) are constants; the host evaluates them once
// with sg_logf and passes them in (P/zoo/neurons/gpea.rs:273-278).
template <class A>
__device__ __forceinline__ bool gpea_step(const A &c, float i_syn, float dt, float ln_na, float ln_k) {
  using namespace gp;
  const float celsius = c.pr(1);
  const float rt = GAS_R * (273.0f + celsius - 9.5f) / CA_FARADAY * 1000.0f;
  const float ena = -rt * ln_na;
  const float ek = rt * ln_k;
  const float inv_cm = c.pr(2), v_thresh = c.pr(3), area = c.pr(4), gnabar = c.pr(5),
              gkdrbar = c.pr(6), gl = c.pr(7), el = c.pr(8), gcatbar = c.pr(9),
              gkcabar = c.pr(10), kca = c.pr(11), vol = c.pr(12), caGain = c.pr(13);
  const float v = c.st(0), m = c.st(1), h = c.st(2), n = c.st(3), p = c.st(4), q = c.st(5),
              cai = c.st(6), r = c.st(7), was_below = c.st(8);
  const float m_inf = gp_sigmoid(v, NA_TH_M, 1.0f / NA_K_M);
  const float m_tau =
      NA_TAU_M0 + NA_TAU_M1 / (1.0f + fast_exp((v - NA_THT_M) * (-1.0f / NA_SIG_M)));
  const float m_new = gp_exp_euler(m, m_inf, m_tau, dt);
  const float h_inf = gp_sigmoid(v, NA_TH_H, 1.0f / NA_K_H);
  const float h_tau =
      gp_tau2(v, NA_TAU_H0, NA_TAU_H1, NA_THT_H1, -1.0f / NA_SIG_H1, NA_THT_H2, 1.0f / NA_SIG_H2);
  const float h_new = gp_exp_euler(h, h_inf, h_tau, dt);
  const float n_inf = gp_sigmoid(v, K_TH_N, 1.0f / K_K_N);
  const float n_tau =
      gp_tau2(v, K_TAU_N0, K_TAU_N1, K_THT_N1, -1.0f / K_SIG_N1, K_THT_N2, 1.0f / K_SIG_N2);
  const float n_new = gp_exp_euler(n, n_inf, n_tau, dt);
  const float p_inf = gp_sigmoid(v, CAT_TH_P, 1.0f / CAT_K_P);
  const float p_tau = gp_tau2(v, CAT_TAU_P0, CAT_TAU_P1, CAT_THT_P1, -1.0f / CAT_SIG_P1,
                              CAT_THT_P2, 1.0f / CAT_SIG_P2);
  const float p_new = gp_exp_euler(p, p_inf, p_tau, dt);
  const float q_inf = gp_sigmoid(v, CAT_TH_Q, 1.0f / CAT_K_Q);
  const float q_tau = gp_tau2(v, CAT_TAU_Q0, CAT_TAU_Q1, CAT_THT_Q1, -1.0f / CAT_SIG_Q1,
                              CAT_THT_Q2, 1.0f / CAT_SIG_Q2);
  const float q_new = gp_exp_euler(q, q_inf, q_tau, dt);
  const float r_inf = gp_sigmoid(cai, AHP_TH_R, 1.0f / AHP_K_R);
  const float r_new = gp_exp_euler(r, r_inf, AHP_TAU_R, dt);

  const float eca_old = -rt * sg_logf(cai / CA_CAO) / 2.0f;
  const float gcat_old = gcatbar * p * p * q;
  const float ica_old = gcat_old * (v - eca_old);
  const float j = -ica_old * area * 1e-14f / (2.0f * CA_FARADAY * vol);
  const float k_ca = caGain * kca;
  const float cai_decay = fast_exp(-dt * k_ca);
  const float cai_new = cai + (1.0f - cai_decay) * (caGain * j / k_ca - cai);
  const float eca = -rt * sg_logf(cai_new / CA_CAO) / 2.0f;

  const float g_na = gnabar * (m_new * m_new * m_new) * h_new;
  const float n2 = n_new * n_new;
  const float g_k = gkdrbar * (n2 * n2);
  const float g_cat = gcatbar * p_new * p_new * q_new;
  const float g_ahp = gkcabar * r_new * r_new;
  const float g_sum = g_na + g_k + g_cat + g_ahp + gl;
  const float g_e_sum = g_na * ena + (g_k + g_ahp) * ek + g_cat * eca + gl * el;
  const float c_over_dt = 1.0f / (inv_cm * dt);
  const float v_new = (c_over_dt * v + i_syn + g_e_sum) / (c_over_dt + g_sum);
  const bool is_above = v_new >= v_thresh;
  const bool spike = is_above && (was_below > 0.0f);  // P/ops/spike.rs:70-74
  c.st(0) = v_new;
  c.st(1) = m_new;
  c.st(2) = h_new;
  c.st(3) = n_new;
  c.st(4) = p_new;
  c.st(5) = q_new;
  c.st(6) = cai_new;
  c.st(7) = r_new;
  c.st(8) = is_above ? 0.0f : 1.0f;
  return spike;
}

// ---- Hodgkin-Huxley, classic RK4 over (V, m, h, n).  The reference HH model
// is a stub (P/zoo/neurons/hh.rs:1-43); rates follow the vtrap form of
// pillars-cuda/kernels/hh.cu:40-63.  i_syn is held over the step.
__device__ __forceinline__ float hh_vtrap(float x, float y) {
  const float r = x / y;
  if (fabsf(r) < 1e-6f) return y - x * 0.5f;
  return x / (sg_expf(r) - 1.0f);
}
struct HHp {
  float c_m, g_na, g_k, g_l, e_na, e_k, e_l, i_ext;
};
__device__ __forceinline__ void hh_deriv(const HHp &P, float v, float m, float h, float n,
                                         float &dv, float &dm, float &dh, float &dn) {
  const float am = 0.1f * hh_vtrap(-(v + 40.0f), 10.0f);
  const float bm = 4.0f * sg_expf(-(v + 65.0f) / 18.0f);
  const float ah = 0.07f * sg_expf(-(v + 65.0f) / 20.0f);
  const float bh = 1.0f / (1.0f + sg_expf(-(v + 35.0f) / 10.0f));
  const float an = 0.01f * hh_vtrap(-(v + 55.0f), 10.0f);
  const float bn = 0.125f * sg_expf(-(v + 65.0f) / 80.0f);
  const float n2 = n * n;
  const float i_na = P.g_na * (m * m * m) * h * (v - P.e_na);
  const float i_k = P.g_k * (n2 * n2) * (v - P.e_k);
  const float i_l = P.g_l * (v - P.e_l);
  dv = (P.i_ext - ((i_na + i_k) + i_l)) / P.c_m;
  dm = am * (1.0f - m) - bm * m;
  dh = ah * (1.0f - h) - bh * h;
  dn = an * (1.0f - n) - bn * n;
}
template <class A> __device__ __forceinline__ bool hh_step(const A &c, float i_syn, float dt) {
  const HHp P{c.pr(1), c.pr(2), c.pr(3), c.pr(4), c.pr(5), c.pr(6), c.pr(7), c.pr(8) + i_syn};
  const float v_th = c.pr(9);
  const float v = c.st(0), m = c.st(1), h = c.st(2), n = c.st(3);
  const float hdt = dt * 0.5f;
  float k1v, k1m, k1h, k1n, k2v, k2m, k2h, k2n, k3v, k3m, k3h, k3n, k4v, k4m, k4h, k4n;
  hh_deriv(P, v, m, h, n, k1v, k1m, k1h, k1n);
  hh_deriv(P, v + hdt * k1v, m + hdt * k1m, h + hdt * k1h, n + hdt * k1n, k2v, k2m, k2h, k2n);
  hh_deriv(P, v + hdt * k2v, m + hdt * k2m, h + hdt * k2h, n + hdt * k2n, k3v, k3m, k3h, k3n);
  hh_deriv(P, v + dt * k3v, m + dt * k3m, h + dt * k3h, n + dt * k3n, k4v, k4m, k4h, k4n);
  const float w = dt / 6.0f;
  const float v_new = v + w * (((k1v + 2.0f * k2v) + 2.0f * k3v) + k4v);
  c.st(0) = v_new;
  c.st(1) = m + w * (((k1m + 2.0f * k2m) + 2.0f * k3m) + k4m);
  c.st(2) = h + w * (((k1h + 2.0f * k2h) + 2.0f * k3h) + k4h);
  c.st(3) = n + w * (((k1n + 2.0f * k2n) + 2.0f * k3n) + k4n);
  return v < v_th && v_new >= v_th;
}

// P/api/net/network/sources.rs:5-14 — stateless Poisson roll (SplitMix64).
__device__ __forceinline__ bool poisson_spike(uint32_t seed, uint32_t stream, uint64_t step,
                                              float p) {
  uint64_t z = ((uint64_t)seed << 32) | (uint64_t)stream;
  z ^= step * 0x9E3779B97F4A7C15ull;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  const float u = (float)(z >> 40) / 16777216.0f;
  return u < p;
}

// ---- Tsodyks-Markram short-term plasticity (P/api/net/push.rs:25-102) ----
// f32 powi as the reference's Rust lowers it for a run-time exponent (the
// compiler runtime's square-and-multiply from the exponent's lowest bit,
// product starting at 1), so that the recovery factors round identically.
__host__ __device__ __forceinline__ float tm_powi(float a, int b) {
  const bool recip = b < 0;
  unsigned e = recip ? 0u - (unsigned)b : (unsigned)b;
  float r = 1.0f;
  while (true) {
    if (e & 1u) r *= a;
    e >>= 1;
    if (e == 0) break;
    a *= a;
  }
  return recip ? 1.0f / r : r;
}
// One spike on one synapse (tm_spike, push.rs:50-81): R and U relax over the
// steps since the last spike, the delivered weight is w * R * U with the
// pre-spike values, then R is depleted and U facilitated.
__host__ __device__ __forceinline__ float tm_spike(float u0, float a_rec, float a_fac, bool fac, float &r,
                                                   float &u, uint32_t &last, float w, unsigned long long step) {
  const unsigned long long el = step > last ? step - last : 0ull;
  const int n = (int)(el < 1000000ull ? el : 1000000ull);
  if (n > 0) {
    r = 1.0f + (r - 1.0f) * tm_powi(a_rec, n);
    if (fac) u = u0 + (u - u0) * tm_powi(a_fac, n);
  }
  last = (uint32_t)step;
  const float scale = r * u;
  r *= 1.0f - u;
  if (fac) u += u0 * (1.0f - u);
  return w * scale;
}

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Counter-based uniform on [0, 1) with 53 random bits: two SplitMix64
// rounds over (seed * golden ratio) ^ (stream << 40) ^ counter.
__host__ __device__ __forceinline__ double hash_uniform01(uint64_t seed, uint32_t stream, uint64_t ctr) {
  const uint64_t key = (seed * 0x9E3779B97F4A7C15ull) ^ ((uint64_t)stream << 40) ^ ctr;
  return (double)(splitmix64(splitmix64(key)) >> 11) * (1.0 / 9007199254740992.0);
}

// Standard normal by the Box-Muller transform in FP64 from the uniforms of
// counters 2c and 2c + 1 (the first mapped to (0, 1]).
__device__ __forceinline__ double hash_std_normal(uint64_t seed, uint32_t stream, uint64_t ctr) {
  const double u1 = 1.0 - hash_uniform01(seed, stream, ctr * 2ull);
  const double u2 = hash_uniform01(seed, stream, ctr * 2ull + 1ull);
  return sqrt(-2.0 * log(u1)) * cos(2.0 * 3.141592653589793 * u2);
}

}  // namespace sg
