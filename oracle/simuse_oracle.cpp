// simuse_oracle.cpp — CPU oracle: a plain C++ restatement of the reference's
// SiMuse simulation step.  TEST INFRASTRUCTURE ONLY (see simuse_oracle.h).
//
// Every function cites the reference file:line it restates, paths relative
// to crates/SiMuse/crates/ (P/ = pillars/src/).  FP32 arithmetic follows the
// reference operation by operation: left-to-right evaluation, no FMA
// contraction (Rust never contracts; this file is built with
// -ffp-contract=off), and explicit fused multiply-add exactly where the
// reference calls mul_add.  Where the reference has no implementation
// (HH with RK4, pair STDP with immediate weight updates, Kuramoto with RK4)
// the formulas here define the behaviour; a templated FP64 twin of every
// model runs the same formulas in double precision.
#include "simuse_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>
#include <thread>

namespace {

thread_local std::string g_err;
int fail(const std::string &m) {
  g_err = m;
  return -1;
}

constexpr uint32_t kSlots = 32;  // P/api/net/graph.rs:33 MAX_DELAY_SLOTS

enum Model { LIF = 1, IZH = 2, GPEA = 3, HH = 4 };
int n_params_of(int m) {
  switch (m) {
    case LIF: return 6;    // P/zoo/neurons/lif.rs:28-39
    case IZH: return 7;    // P/zoo/neurons/izhikevich.rs:50-63
    case GPEA: return 14;  // P/zoo/neurons/gpea.rs:231-258
    case HH: return 10;    // dt c_m g_na g_k g_l e_na e_k e_l i_bias v_thresh
  }
  return -1;
}
int n_state_of(int m) {
  switch (m) {
    case LIF: return 2;
    case IZH: return 3;
    case GPEA: return 9;
    case HH: return 4;  // v m h n
  }
  return -1;
}
bool clamps_input(int m) {
  // P/core/exec/population.rs:69-86: CLAMP_I_SYN defaults to true; GPEA is
  // #[no_clamp] (P/zoo/neurons/gpea.rs:210).  HH here is a conductance model
  // and is defined without the clamp as well.
  return m == LIF || m == IZH;
}

// ---------------------------------------------------------------------------
// Math
// ---------------------------------------------------------------------------

// P/math/fast_exp.rs:23-68, the fused (x86_64 + fma) flavour.
float fast_exp_f(float x) {
  const float log2e = 1.44269504088896340736f;
  float t = x * log2e;
  float tf = std::floor(t);
  int n;
  if (std::isnan(tf)) n = 0;
  else if (tf >= 2147483647.0f) n = 2147483647;
  else if (tf <= -2147483648.0f) n = (-2147483647 - 1);
  else n = (int)tf;
  float f = t - (float)n;
  const float c1 = 0.693147180559945309417f;
  const float c2 = 0.2402265f;
  const float c3 = 0.05550411f;
  const float c4 = 0.009618129f;
  const float c5 = 0.001333356f;
  const float c6 = 0.0001540353f;
  float poly = std::fma(c6, f, c5);
  poly = std::fma(poly, f, c4);
  poly = std::fma(poly, f, c3);
  poly = std::fma(poly, f, c2);
  poly = std::fma(poly, f, c1);
  poly = std::fma(poly, f, 1.0f);
  if (n < -126) return 0.0f;
  if (n > 127) return INFINITY;
  uint32_t bits = (uint32_t)(n + 127) << 23;
  float s;
  std::memcpy(&s, &bits, 4);
  return s * poly;
}

// Exponential used by the HH model in FP32 (shared definition with the CUDA
// kernel: Cody-Waite reduction by ln 2 split into a short high part and a
// low part, degree-7 Taylor polynomial of e^r on |r| <= ln2/2, exponent
// scaling by bit construction).  Written from the mathematics.
float sg_expf(float x) {
  if (x > 88.0f) x = 88.0f;
  if (x < -87.0f) x = -87.0f;
  const float log2e = 1.44269504088896340736f;
  const float ln2_hi = 0.693145751953125f;
  const float ln2_lo = 1.428606820309417232e-6f;
  float k = std::nearbyint(x * log2e);
  float r = std::fma(-k, ln2_hi, x);
  r = std::fma(-k, ln2_lo, r);
  float p = 1.0f / 5040.0f;
  p = std::fma(p, r, 1.0f / 720.0f);
  p = std::fma(p, r, 1.0f / 120.0f);
  p = std::fma(p, r, 1.0f / 24.0f);
  p = std::fma(p, r, 1.0f / 6.0f);
  p = std::fma(p, r, 0.5f);
  p = std::fma(p, r, 1.0f);
  p = std::fma(p, r, 1.0f);
  int ki = (int)k;
  // 2^k split in two factors so that k in [-126, 127] never leaves the
  // normal range of either factor.
  int k1 = ki / 2, k2 = ki - k1;
  uint32_t b1 = (uint32_t)(k1 + 127) << 23, b2 = (uint32_t)(k2 + 127) << 23;
  float s1, s2;
  std::memcpy(&s1, &b1, 4);
  std::memcpy(&s2, &b2, 4);
  return (p * s1) * s2;
}

// Natural log used by the GPEA calcium Nernst potential in FP32, the same
// definition as the CUDA kernel's: x = m * 2^k, m in [sqrt(1/2), sqrt(2)),
// ln m = 2 atanh((m - 1)/(m + 1)) by its series to s^25 (Abramowitz & Stegun
// 4.1.27) in FP64, plus k ln 2 (split in a high and a low part), rounded once
// to FP32: correctly rounded over every float in [1e-12, 1e6].  The
// reference's f32::ln is the platform libm logf, which (glibc) differs from
// the correctly rounded value by one unit in the last place on about 0.07% of
// those floats; this restatement takes the correctly rounded value so that
// the device can reproduce it.
float sg_logf(float x) {
  uint32_t b;
  std::memcpy(&b, &x, 4);
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (b >= 0x7f800000u) return x;
  int k = 0;
  if (b < 0x00800000u) {
    x = x * 16777216.0f;
    std::memcpy(&b, &x, 4);
    k = -24;
  }
  k += (int)(b >> 23) - 127;
  const uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
  float mf;
  std::memcpy(&mf, &mb, 4);
  double m = (double)mf;
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    k += 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double z = s * s;
  double p = 1.0 / 25.0;
  const double inv[12] = {1.0 / 23.0, 1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0,
                          1.0 / 11.0, 1.0 / 9.0,  1.0 / 7.0,  1.0 / 5.0,  1.0 / 3.0,  1.0};
  for (double c : inv) p = p * z + c;
  const double lm = (2.0 * s) * p;
  const double ln2_hi = 6.93147180369123816490e-01, ln2_lo = 1.90821492927058770002e-10;
  return (float)((double)k * ln2_hi + ((double)k * ln2_lo + lm));
}

template <typename T> struct M;
template <> struct M<float> {
  static float fexp(float x) { return fast_exp_f(x); }  // GPEA, STDP decay
  static float hexp(float x) { return sg_expf(x); }     // HH rates
  static float ln(float x) { return sg_logf(x); }      // GPEA Nernst
  static float fma(float a, float b, float c) { return std::fma(a, b, c); }
};
template <> struct M<double> {
  static double fexp(double x) { return std::exp(x); }
  static double hexp(double x) { return std::exp(x); }
  static double ln(double x) { return std::log(x); }
  static double fma(double a, double b, double c) { return std::fma(a, b, c); }
};

// Receptor kinetics of SynapticBrain (pillars-connectome/src/synaptic.rs).
// Decay time constant (ms) and reversal potential (mV) per receptor code,
// P/kernels/synapse/receptor.rs:71-100: 0 AMPA, 1 NMDA, 2 GABA_A, 3 GABA_B,
// 4 nAChR, 5 GluCl, 6 mAChR; any other code is AMPA (:103-115).
constexpr int kReceptors = 7;
constexpr float kRecTau[kReceptors] = {2.0f, 50.0f, 10.0f, 200.0f, 3.0f, 5.0f, 150.0f};
constexpr float kRecErev[kReceptors] = {0.0f, 0.0f, -65.0f, -90.0f, 0.0f, -70.0f, -90.0f};
inline int receptor_of(uint8_t code) { return code < kReceptors ? code : 0; }

// P/kernels/synapse/receptor.rs:126-131 nmda_mg_block:
// 1 / (1 + 0.33 exp(clamp(-0.06 v, -10, 10))) with the project's fast_exp
// (the SIMD form of :135-143 gives the same bits).
template <typename T> T nmda_mg_block(T v) {
  T a = (T)-0.06f * v;
  if (a < (T)-10.0f) a = (T)-10.0f;
  if (a > (T)10.0f) a = (T)10.0f;
  return (T)1.0f / ((T)1.0f + (T)0.33f * M<T>::fexp(a));
}

// DecayFactors::new(dt), P/kernels/synapse/kinetics.rs:27-38: fast_exp(-dt/tau).
template <typename T> void receptor_factors(float dt, T f[kReceptors]) {
  for (int r = 0; r < kReceptors; ++r) f[r] = M<T>::fexp(-(T)dt / (T)kRecTau[r]);
}

// One neuron of SynapticKinetics::compute_currents, P/kernels/synapse/
// kinetics.rs:159-206: from zero, over the receptors in code order,
// cur += g_eff (E_rev - v), g_eff = g * mg_block(v) for NMDA, g otherwise.
// g[r] is the neuron's conductance of receptor r.
template <typename T> T receptor_current(const T g[kReceptors], T v) {
  const T b = nmda_mg_block(v);
  T cur = (T)0;
  for (int r = 0; r < kReceptors; ++r) {
    const T ge = r == 1 ? g[r] * b : g[r];
    cur += ge * ((T)kRecErev[r] - v);
  }
  return cur;
}

// P/api/net/network/sources.rs:5-14
bool poisson_spike(uint32_t seed, uint32_t stream, uint64_t step, float p) {
  uint64_t z = ((uint64_t)seed << 32) | (uint64_t)stream;
  z ^= step * 0x9E3779B97F4A7C15ull;
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  float u = (float)(z >> 40) / (float)(1ull << 24);
  return u < p;
}

// ---------------------------------------------------------------------------
// Neuron models (one neuron, SoA accessors)
// ---------------------------------------------------------------------------

template <typename T> struct Cols {
  T *s;
  const T *p;
  uint32_t cap, i;
  T &st(int c) const { return s[(size_t)c * cap + i]; }
  T pr(int c) const { return p[(size_t)c * cap + i]; }
};

// P/zoo/neurons/lif.rs:47-78
template <typename T> bool lif_step(const Cols<T> &c, T i_syn, T dt) {
  const T zero = 0;
  T v = c.st(0), refr = c.st(1);
  const T inv_tau = c.pr(1), v_rest = c.pr(2), v_th = c.pr(3), v_reset = c.pr(4),
          tau_ref = c.pr(5);
  bool is_refr = refr > zero;
  T dv = ((v_rest - v) + i_syn) * inv_tau * dt;
  T v_new = v + dv;
  bool spike = is_refr ? false : (v_new >= v_th);
  T v_final = spike ? v_reset : v_new;
  c.st(0) = is_refr ? v : v_final;
  T refr_dec = refr - dt;
  T refr_set = spike ? tau_ref : refr_dec;
  c.st(1) = std::fmax(refr_set, zero);
  return spike;
}

// P/zoo/neurons/izhikevich.rs:71-125
template <typename T> bool izh_step(const Cols<T> &c, T i_syn, T dt) {
  const T zero = 0;
  T vs = c.st(0), u = c.st(1), refr = c.st(2);
  const T a = c.pr(1), b = c.pr(2), cc = c.pr(3), d = c.pr(4), tau_ref = c.pr(5),
          v_th = c.pr(6);
  bool is_refr = refr > zero;
  T v = is_refr ? cc : vs;
  T half_dt = dt * (T)0.5;
  const T c04 = (T)0.04f, c5 = 5, c140 = 140;
  T v_poly1 = v * (c04 * v + c5);
  T dv1 = (v_poly1 + c140 - u + i_syn) * half_dt;
  T v_mid = v + dv1;
  T v_poly2 = v_mid * (c04 * v_mid + c5);
  T dv2 = (v_poly2 + c140 - u + i_syn) * half_dt;
  T dv_total = is_refr ? zero : dv1 + dv2;
  T v_new = v + dv_total;
  T du = a * (b * v - u) * dt;
  T u_new = is_refr ? u : u + du;
  bool spike = v_new >= v_th;
  c.st(0) = spike ? cc : v_new;
  c.st(1) = spike ? u_new + d : u_new;
  T refr_dec = refr - dt;
  T refr_set = spike ? tau_ref : refr_dec;
  c.st(2) = std::fmax(refr_set, zero);
  return spike;
}

// P/zoo/neurons/gpea.rs:53-123 constants, :129-179 helpers, :266-360 step.
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
constexpr float CA_FARADAY = 96485.0f;
constexpr float NA_NAI = 10.0f, NA_NAO = 140.0f, K_KI = 140.0f, K_KO = 5.0f, CA_CAO = 2.0f;
constexpr float GAS_R = 8.31441f;
}  // namespace gp

template <typename T> T g_sigmoid(T x, float th, float k) {
  return (T)1 / ((T)1 + M<T>::fexp((x - (T)th) * (T)(1.0f / k)));
}
template <typename T> T g_exp_euler(T x, T x_inf, T tau, T dt) {
  T decay = M<T>::fexp(-dt / tau);
  return M<T>::fma(decay, x - x_inf, x_inf);
}
template <typename T> T g_tau2(T v, float t0, float t1, float th1, float s1, float th2, float s2) {
  T e1 = M<T>::fexp((v - (T)th1) * (T)(-1.0f / s1));
  T e2 = M<T>::fexp((-(v - (T)th2)) * (T)(1.0f / s2));
  return (T)t0 + (T)t1 / (e1 + e2);
}

template <typename T> bool gpea_step(const Cols<T> &c, T i_syn, T dt) {
  using namespace gp;
  T celsius = c.pr(1), inv_cm = c.pr(2), v_thresh = c.pr(3), area = c.pr(4), gnabar = c.pr(5),
    gkdrbar = c.pr(6), gl = c.pr(7), el = c.pr(8), gcatbar = c.pr(9), gkcabar = c.pr(10),
    kca = c.pr(11), vol = c.pr(12), caGain = c.pr(13);
  T rt = (T)GAS_R * ((T)273.0f + celsius - (T)9.5f) / (T)CA_FARADAY * (T)1000.0f;
  T ena = -rt * M<T>::ln((T)NA_NAI / (T)NA_NAO);
  T ek = rt * M<T>::ln((T)K_KO / (T)K_KI);
  T v = c.st(0), m = c.st(1), h = c.st(2), n = c.st(3), p = c.st(4), q = c.st(5), cai = c.st(6),
    r = c.st(7), was_below = c.st(8);

  T m_inf = g_sigmoid(v, NA_TH_M, NA_K_M);
  T m_tau;
  {
    T denom = (T)1 + M<T>::fexp((v - (T)NA_THT_M) * (T)(-1.0f / NA_SIG_M));
    m_tau = (T)NA_TAU_M0 + (T)NA_TAU_M1 / denom;
  }
  T m_new = g_exp_euler(m, m_inf, m_tau, dt);
  T h_inf = g_sigmoid(v, NA_TH_H, NA_K_H);
  T h_tau = g_tau2(v, NA_TAU_H0, NA_TAU_H1, NA_THT_H1, NA_SIG_H1, NA_THT_H2, NA_SIG_H2);
  T h_new = g_exp_euler(h, h_inf, h_tau, dt);
  T n_inf = g_sigmoid(v, K_TH_N, K_K_N);
  T n_tau = g_tau2(v, K_TAU_N0, K_TAU_N1, K_THT_N1, K_SIG_N1, K_THT_N2, K_SIG_N2);
  T n_new = g_exp_euler(n, n_inf, n_tau, dt);
  T p_inf = g_sigmoid(v, CAT_TH_P, CAT_K_P);
  T p_tau = g_tau2(v, CAT_TAU_P0, CAT_TAU_P1, CAT_THT_P1, CAT_SIG_P1, CAT_THT_P2, CAT_SIG_P2);
  T p_new = g_exp_euler(p, p_inf, p_tau, dt);
  T q_inf = g_sigmoid(v, CAT_TH_Q, CAT_K_Q);
  T q_tau = g_tau2(v, CAT_TAU_Q0, CAT_TAU_Q1, CAT_THT_Q1, CAT_SIG_Q1, CAT_THT_Q2, CAT_SIG_Q2);
  T q_new = g_exp_euler(q, q_inf, q_tau, dt);
  T r_inf = g_sigmoid(cai, AHP_TH_R, AHP_K_R);
  T r_new = g_exp_euler(r, r_inf, (T)AHP_TAU_R, dt);

  T eca_old = -rt * M<T>::ln(cai / (T)CA_CAO) / (T)2.0f;
  T gcat_old = gcatbar * p * p * q;
  T ica_old = gcat_old * (v - eca_old);
  T j = -ica_old * area * (T)1e-14f / ((T)2.0f * (T)CA_FARADAY * vol);
  T k_ca = caGain * kca;
  T cai_decay = M<T>::fexp(-dt * k_ca);
  T cai_new = cai + ((T)1 - cai_decay) * (caGain * j / k_ca - cai);
  T eca = -rt * M<T>::ln(cai_new / (T)CA_CAO) / (T)2.0f;

  T g_na = gnabar * (m_new * m_new * m_new) * h_new;
  T n2 = n_new * n_new;
  T g_k = gkdrbar * (n2 * n2);
  T g_cat = gcatbar * p_new * p_new * q_new;
  T g_ahp = gkcabar * r_new * r_new;
  T g_leak = gl;
  T g_sum = g_na + g_k + g_cat + g_ahp + g_leak;
  T g_e_sum = g_na * ena + (g_k + g_ahp) * ek + g_cat * eca + g_leak * el;
  T c_over_dt = (T)1 / (inv_cm * dt);
  T v_new = (c_over_dt * v + i_syn + g_e_sum) / (c_over_dt + g_sum);
  bool is_above = v_new >= v_thresh;
  bool spike = is_above && (was_below > (T)0);  // P/ops/spike.rs:70-74
  c.st(0) = v_new;
  c.st(1) = m_new;
  c.st(2) = h_new;
  c.st(3) = n_new;
  c.st(4) = p_new;
  c.st(5) = q_new;
  c.st(6) = cai_new;
  c.st(7) = r_new;
  c.st(8) = is_above ? (T)0 : (T)1;
  return spike;
}

// Hodgkin-Huxley with classic RK4 over (V, m, h, n).  The reference's HH
// model is a stub (P/zoo/neurons/hh.rs:1-43); the rate functions follow the
// reference CUDA kernel's vtrap form (pillars-cuda/kernels/hh.cu:40-63).
// The synaptic current i_syn is held fixed over the step (the reference
// computes conductance currents from V at the start of the step,
// P/api/net/network/step.rs:36-70).
template <typename T> T hh_vtrap(T x, T y) {
  T r = x / y;
  if (std::fabs(r) < (T)1e-6f) return y - x * (T)0.5f;
  return x / (M<T>::hexp(r) - (T)1);
}
template <typename T> struct HHp { T c_m, g_na, g_k, g_l, e_na, e_k, e_l, i_ext; };
template <typename T>
void hh_deriv(const HHp<T> &P, T v, T m, T h, T n, T &dv, T &dm, T &dh, T &dn) {
  T am = (T)0.1f * hh_vtrap(-(v + (T)40), (T)10);
  T bm = (T)4 * M<T>::hexp(-(v + (T)65) / (T)18);
  T ah = (T)0.07f * M<T>::hexp(-(v + (T)65) / (T)20);
  T bh = (T)1 / ((T)1 + M<T>::hexp(-(v + (T)35) / (T)10));
  T an = (T)0.01f * hh_vtrap(-(v + (T)55), (T)10);
  T bn = (T)0.125f * M<T>::hexp(-(v + (T)65) / (T)80);
  T n2 = n * n;
  T i_na = P.g_na * (m * m * m) * h * (v - P.e_na);
  T i_k = P.g_k * (n2 * n2) * (v - P.e_k);
  T i_l = P.g_l * (v - P.e_l);
  dv = (P.i_ext - ((i_na + i_k) + i_l)) / P.c_m;
  dm = am * ((T)1 - m) - bm * m;
  dh = ah * ((T)1 - h) - bh * h;
  dn = an * ((T)1 - n) - bn * n;
}
template <typename T> bool hh_step(const Cols<T> &c, T i_syn, T dt) {
  HHp<T> P{c.pr(1), c.pr(2), c.pr(3), c.pr(4), c.pr(5), c.pr(6), c.pr(7), c.pr(8) + i_syn};
  T v_th = c.pr(9);
  T v = c.st(0), m = c.st(1), h = c.st(2), n = c.st(3);
  T hdt = dt * (T)0.5f;
  T k1v, k1m, k1h, k1n, k2v, k2m, k2h, k2n, k3v, k3m, k3h, k3n, k4v, k4m, k4h, k4n;
  hh_deriv(P, v, m, h, n, k1v, k1m, k1h, k1n);
  hh_deriv(P, v + hdt * k1v, m + hdt * k1m, h + hdt * k1h, n + hdt * k1n, k2v, k2m, k2h, k2n);
  hh_deriv(P, v + hdt * k2v, m + hdt * k2m, h + hdt * k2h, n + hdt * k2n, k3v, k3m, k3h, k3n);
  hh_deriv(P, v + dt * k3v, m + dt * k3m, h + dt * k3h, n + dt * k3n, k4v, k4m, k4h, k4n);
  T w = dt / (T)6;
  T v_new = v + w * (((k1v + (T)2 * k2v) + (T)2 * k3v) + k4v);
  c.st(0) = v_new;
  c.st(1) = m + w * (((k1m + (T)2 * k2m) + (T)2 * k3m) + k4m);
  c.st(2) = h + w * (((k1h + (T)2 * k2h) + (T)2 * k3h) + k4h);
  c.st(3) = n + w * (((k1n + (T)2 * k2n) + (T)2 * k3n) + k4n);
  return v < v_th && v_new >= v_th;
}

// ---------------------------------------------------------------------------
// Network
// ---------------------------------------------------------------------------

template <typename T> struct Pop {
  int model;
  uint32_t n, cap, np, ns;
  std::vector<T> params, state;  // SoA [col][cap], P/core/exec/population.rs:106-127
};

struct EdgeIn {
  uint32_t pre, post;
  float w;
  uint8_t d, st, flags, pt;  // pt: short-term plasticity profile id (0 = none)
};

// P/api/net/push.rs:25-35 PlastRtProfile: Tsodyks-Markram constants for one dt
struct TmProf {
  float u0, a_rec, a_fac;
  bool fac;
};

// f32 powi as Rust lowers it for a run-time exponent (the compiler runtime's
// __powisf2): square-and-multiply from the exponent's lowest bit, the
// product starting at 1, reciprocal for a negative exponent.
static float powi_f32(float a, int b) {
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

// P/api/net/push.rs:50-81 tm_spike: lazy exponential recovery over the steps
// since the last spike, deliver weight * R * U with the pre-spike R and U,
// then deplete R and facilitate U.
static float tm_spike(const TmProf &p, float &r, float &u, uint32_t &last, float w, uint64_t step) {
  const uint64_t el = step > last ? step - last : 0;
  const int n = (int)std::min<uint64_t>(el, 1000000);
  if (n > 0) {
    const float ar = powi_f32(p.a_rec, n);
    r = 1.0f + (r - 1.0f) * ar;
    if (p.fac) {
      const float af = powi_f32(p.a_fac, n);
      u = p.u0 + (u - p.u0) * af;
    }
  }
  last = (uint32_t)step;
  const float scale = r * u;
  r *= 1.0f - u;
  if (p.fac) u += p.u0 * (1.0f - u);
  return w * scale;
}

// P/api/net/network/step.rs:206-298 KinKind: a kinetic synapse's per-step
// constants (f32, from the host libm).  kind 0 ExpOne {a_decay}, 1 ExpTwo
// {a_rise, a_decay, norm}, 2 Alpha {r, e*(dt/tau)*r}, 3 ExpThree {a_rise,
// a_decay1, a_decay2, wf1, wf2, k_a, gbase1, gbase2}
struct Kin {
  int kind;
  float erev;
  float c[8];
};

// P/api/net/synapse.rs:296-305 exp_waveform_factor (NeuroML waveformFactor)
static float waveform_factor(float tr, float td) {
  const float t_peak = (tr * td) / (td - tr) * std::log(td / tr);
  const float h = std::exp(-t_peak / td) - std::exp(-t_peak / tr);
  return 1.0f / h;
}

template <typename T> struct Src {
  float p;
  uint32_t seed;
  std::vector<uint32_t> post;
  std::vector<T> w;
  std::vector<uint8_t> d, st;
  // Tsodyks-Markram profile per outgoing synapse (0 none) and its state
  // R, U, last spike step (P/api/net/network/sources.rs:20-31, core.rs:372-378)
  std::vector<uint8_t> pt;
  std::vector<float> r, u;
  std::vector<uint32_t> last;
};

struct Stdp {
  bool on = false;
  float dt, tau_pre, tau_post, a_plus, a_minus, w_min, w_max;
};

// P/api/learn/brain.rs:17-141 StdpConfig + Brain state (dopamine-modulated
// eligibility learning over the network's own synapses, CSR order)
struct Learn {
  bool on = false;
  float dt, tau_pre, tau_post, tau_e, a_ltp, a_ltd, lr, w_min, w_max;
  uint64_t t = 0;
  std::vector<float> tp, tq, elig;
  std::vector<uint64_t> last, stamp;
  std::vector<uint32_t> in_ptr, in_edge, pre_of;
  std::vector<std::pair<uint32_t, float>> events;
  std::vector<float> baked;  // snapshot of the weights (brain.rs:344-347)
  // spikes of [lo0, hi0) and [lo1, hi1) counted since the step call began
  // (pillars-wgpu/src/network.rs:902-955 motor sums)
  uint64_t motor_lo[2] = {0, 0}, motor_hi[2] = {0, 0};
  uint32_t motor[2] = {0, 0};
};

struct NetBase {
  virtual ~NetBase() {}
};

template <typename T> struct Net : NetBase {
  std::vector<Pop<T>> pops;
  std::vector<uint32_t> offsets{0};
  uint64_t total = 0;
  bool built = false;
  std::vector<EdgeIn> edges;
  std::vector<uint32_t> row_ptr, col;
  std::vector<T> w;
  std::vector<uint8_t> d, st, plastic, pt;
  std::vector<TmProf> tm;           // short-term plasticity profiles (id - 1)
  std::vector<float> tm_r, tm_u;    // per edge (CSR order): R, U
  std::vector<uint32_t> tm_last;    //   and the step of its last spike
  std::vector<Kin> kin;
  std::vector<T> g;     // [nk][N] kinetic conductances
  // SynapticBrain mode: the edges' syn_types are receptor codes, every
  // spike jumps the conductance rg[receptor][post] at once (no delay), and
  // each step decays them and adds their ohmic current to the input
  bool receptor = false;
  float rec_dt = 0.0f;
  std::vector<T> rg;    // [7][N]
  std::vector<T> ring;  // [1 + nk][32][N]
  std::vector<Src<T>> srcs;
  uint64_t step = 0, events = 0;
  std::vector<T> i_in, v_scr, scratch;
  std::vector<int32_t> spikes;
  std::vector<uint32_t> active;
  Stdp stdp;
  std::vector<T> x_pre, x_post;
  std::vector<uint32_t> in_ptr, in_edge, in_pre;  // CSC of plastic edges
  double drift = 0.0;
  Learn learn;

  T *ring_slot(uint32_t r, uint32_t slot) { return &ring[((size_t)r * kSlots + slot) * total]; }
};

// P/api/net/graph.rs:104-206 from_triplets_with_types: validate, sort by pre,
// count, prefix-sum a u32 row_ptr, place.  The reference sorts by pre with an
// unstable sort, so the order inside a row is not part of its contract; here
// a row is ordered by post, stably (repeated (pre, post) synapses keep
// insertion order, and with it every ring cell's summation order).
template <typename T> int build_csr(Net<T> &net) {
  const uint64_t E = net.edges.size();
  const uint64_t N = net.total;
  std::vector<uint64_t> counts(N + 1, 0);
  for (auto &e : net.edges) counts[e.pre]++;
  net.row_ptr.assign(N + 1, 0);
  uint64_t cum = 0;
  for (uint64_t i = 0; i < N; ++i) {
    if (cum > 0xFFFFFFFFull) return fail("SparseGraph: too many synapses for a u32 CSR row_ptr");
    net.row_ptr[i] = (uint32_t)cum;
    cum += counts[i];
  }
  if (cum > 0xFFFFFFFFull) return fail("SparseGraph: too many synapses for a u32 CSR row_ptr");
  net.row_ptr[N] = (uint32_t)cum;
  net.col.assign(E, 0);
  net.w.assign(E, 0);
  net.d.assign(E, 0);
  net.st.assign(E, 0);
  net.plastic.assign(E, 0);
  net.pt.assign(E, 0);
  std::vector<uint64_t> cursor(net.row_ptr.begin(), net.row_ptr.end() - 1);
  for (auto &e : net.edges) {
    uint64_t pos = cursor[e.pre]++;
    net.col[pos] = e.post;
    net.w[pos] = (T)e.w;
    net.d[pos] = e.d;
    net.st[pos] = e.st;
    net.plastic[pos] = e.flags & 1;
    net.pt[pos] = e.pt;
  }
  net.edges.clear();
  net.edges.shrink_to_fit();
  std::vector<uint64_t> idx;
  for (uint64_t i = 0; i < N; ++i) {
    const uint64_t a = net.row_ptr[i], b = net.row_ptr[i + 1];
    bool sorted = true;
    for (uint64_t e = a + 1; e < b && sorted; ++e) sorted = net.col[e - 1] <= net.col[e];
    if (sorted) continue;
    idx.resize(b - a);
    for (uint64_t k = 0; k < b - a; ++k) idx[k] = a + k;
    std::stable_sort(idx.begin(), idx.end(), [&](uint64_t x, uint64_t y) { return net.col[x] < net.col[y]; });
    auto permute = [&](auto &v) {
      using V = typename std::decay_t<decltype(v)>::value_type;
      std::vector<V> tmp(b - a);
      for (uint64_t k = 0; k < b - a; ++k) tmp[k] = v[idx[k]];
      std::copy(tmp.begin(), tmp.end(), v.begin() + a);
    };
    permute(net.col);
    permute(net.w);
    permute(net.d);
    permute(net.st);
    permute(net.plastic);
    permute(net.pt);
  }
  return 0;
}

template <typename T> void alloc_runtime(Net<T> &net) {
  const size_t N = net.total;
  // P/api/net/network/build.rs:69-84: R = 1, U = U0 of the edge's profile, last = 0
  if (!net.tm.empty()) {
    const size_t E = net.col.size();
    net.tm_r.assign(E, 1.0f);
    net.tm_u.assign(E, 0.0f);
    net.tm_last.assign(E, 0);
    for (size_t e = 0; e < E; ++e)
      if (net.pt[e]) net.tm_u[e] = net.tm[net.pt[e] - 1].u0;
  }
  net.ring.assign((1 + net.kin.size()) * kSlots * N, (T)0);
  net.g.assign(net.kin.size() * 3 * N, (T)0);  // up to three state arrays per profile
  if (net.receptor) net.rg.assign((size_t)kReceptors * N, (T)0);
  net.i_in.assign(N, (T)0);
  net.v_scr.assign(N, (T)0);
  net.scratch.assign(N, (T)0);
  net.spikes.assign(N, 0);
  net.active.reserve(N / 20 + 8);
  if (net.stdp.on) {
    net.x_pre.assign(N, (T)0);
    net.x_post.assign(N, (T)0);
    // in-edges of plastic synapses, grouped by post (Brain keeps in_edges,
    // P/api/learn/brain.rs:79-80,113-118)
    std::vector<uint64_t> cnt(N + 1, 0);
    for (uint64_t pre = 0; pre < N; ++pre)
      for (uint64_t e = net.row_ptr[pre]; e < net.row_ptr[pre + 1]; ++e)
        if (net.plastic[e]) cnt[net.col[e]]++;
    net.in_ptr.assign(N + 1, 0);
    uint64_t c = 0;
    for (uint64_t i = 0; i < N; ++i) {
      net.in_ptr[i] = (uint32_t)c;
      c += cnt[i];
    }
    net.in_ptr[N] = (uint32_t)c;
    net.in_edge.assign(c, 0);
    net.in_pre.assign(c, 0);
    std::vector<uint64_t> cur(net.in_ptr.begin(), net.in_ptr.end() - 1);
    for (uint64_t pre = 0; pre < N; ++pre)
      for (uint64_t e = net.row_ptr[pre]; e < net.row_ptr[pre + 1]; ++e)
        if (net.plastic[e]) {
          uint64_t k = cur[net.col[e]]++;
          net.in_edge[k] = (uint32_t)e;
          net.in_pre[k] = (uint32_t)pre;
        }
  }
  net.built = true;
}

int g_threads = 1;

// P/api/net/network/step.rs:18-189 Network::step, then (when configured) the
// pair-STDP update of the plastic weights.
// A step in two halves, so that a network split across processes can
// exchange the spikes of its external populations (neurons simulated by
// another rank) between them: the first half reads the ring slot and
// updates the populations simulated here; the second compacts every spike
// (local and external), pushes, rolls the sources and learns.
template <typename T> void net_step_begin(Net<T> &net) {
  const size_t N = net.total;
  if (N == 0) return;
  const uint32_t slot = (uint32_t)(net.step % kSlots);
  // 1-2. read the current slot into i_in, clear it (step.rs:27-34)
  T *rs = net.ring_slot(0, slot);
  std::memcpy(net.i_in.data(), rs, N * sizeof(T));
  std::memset(rs, 0, N * sizeof(T));
  // 2b. kinetic synapses (step.rs:36-70; ExpOne at :338-345)
  if (!net.kin.empty()) {
    for (size_t p = 0; p < net.pops.size(); ++p) {
      auto &pop = net.pops[p];
      for (uint32_t i = 0; i < pop.n; ++i) net.v_scr[net.offsets[p] + i] = pop.state[i];
    }
    for (size_t k = 0; k < net.kin.size(); ++k) {
      T *ks = net.ring_slot((uint32_t)k + 1, slot);
      std::memcpy(net.scratch.data(), ks, N * sizeof(T));
      std::memset(ks, 0, N * sizeof(T));
      const Kin &K = net.kin[k];
      const T erev = (T)K.erev;
      T c[8];
      for (int q = 0; q < 8; ++q) c[q] = (T)K.c[q];
      T *s0 = &net.g[(k * 3 + 0) * N], *s1 = &net.g[(k * 3 + 1) * N], *s2 = &net.g[(k * 3 + 2) * N];
      for (size_t i = 0; i < N; ++i) {  // step.rs:336-398
        const T j = net.scratch[i], dv = erev - net.v_scr[i];
        if (K.kind == 0) {  // ExpOne: g
          const T gn = s0[i] * c[0] + j;
          s0[i] = gn;
          net.i_in[i] += gn * dv;
        } else if (K.kind == 1) {  // ExpTwo: g (decay), x (rise)
          const T gn = s0[i] * c[1] + j;
          const T xn = s1[i] * c[0] + j;
          s0[i] = gn;
          s1[i] = xn;
          net.i_in[i] += c[2] * (gn - xn) * dv;
        } else if (K.kind == 2) {  // Alpha: g, a
          const T a_old = s1[i];
          const T an = a_old * c[0] + j;
          const T gn = s0[i] * c[0] + c[1] * a_old;
          s0[i] = gn;
          s1[i] = an;
          net.i_in[i] += gn * dv;
        } else {  // ExpThree: a (rise), b, c (decays)
          const T an = s0[i] * c[0] + j * c[5];
          const T bn = s1[i] * c[1] + j * c[3];
          const T cn = s2[i] * c[2] + j * c[4];
          s0[i] = an;
          s1[i] = bn;
          s2[i] = cn;
          const T cur = c[6] * (bn - an) + c[7] * (cn - an);
          net.i_in[i] += cur * dv;
        }
      }
    }
  }
  // 2c. SynapticBrain::step (pillars-connectome/src/synaptic.rs:94-112):
  // decay every conductance by its factor (P/kernels/synapse/kinetics.rs:
  // 112-147; factors fast_exp(-dt/tau), :27-38), then I_syn = sum over the
  // receptors in code order of g_eff (E_rev - V) from zero, NMDA's g scaled
  // by the Mg block of the pre-step V (:159-206), and i_in = I_syn + the
  // external input (here the step's injected current).
  if (net.receptor) {
    T f[kReceptors];
    receptor_factors(net.rec_dt, f);
    for (size_t p = 0; p < net.pops.size(); ++p) {
      auto &pop = net.pops[p];
      for (uint32_t i = 0; i < pop.n; ++i) net.v_scr[net.offsets[p] + i] = pop.state[i];
    }
    for (size_t i = 0; i < N; ++i) {
      T g[kReceptors];
      for (int r = 0; r < kReceptors; ++r) {
        T &gr = net.rg[(size_t)r * N + i];
        gr = gr * f[r];
        g[r] = gr;
      }
      net.i_in[i] = receptor_current(g, net.v_scr[i]) + net.i_in[i];
    }
  }
  // 3. populations (P/core/exec/population.rs:284-465).  dt is param column 0
  // of neuron 0, broadcast to the population (:307,:361).
  for (size_t p = 0; p < net.pops.size(); ++p) {
    auto &pop = net.pops[p];
    if (pop.n == 0 || pop.model == 0) continue;  // model 0: external, spikes set by the exchange
    const T dt = pop.params[0];
    const bool clamp = clamps_input(pop.model);
    const uint32_t off = net.offsets[p];
    for (uint32_t i = 0; i < pop.n; ++i) {
      T x = net.i_in[off + i];
      if (clamp) x = std::fmin(std::fmax(x, (T)-100.0f), (T)100.0f);
      Cols<T> c{pop.state.data(), pop.params.data(), pop.cap, i};
      bool s = false;
      switch (pop.model) {
        case LIF: s = lif_step(c, x, dt); break;
        case IZH: s = izh_step(c, x, dt); break;
        case GPEA: s = gpea_step(c, x, dt); break;
        case HH: s = hh_step(c, x, dt); break;
      }
      net.spikes[off + i] = s ? 1 : 0;
    }
  }
}

template <typename T> void net_step_end(Net<T> &net) {
  const size_t N = net.total;
  if (N == 0) {
    net.step++;
    return;
  }
  // 4. compaction, ascending (P/api/net/compact.rs:30-61)
  net.active.clear();
  for (size_t i = 0; i < N; ++i)
    if (net.spikes[i] != 0) net.active.push_back((uint32_t)i);
  // 5. push (P/api/net/push.rs:126-173; the rayon variant :184-237 collects
  // (post, slot, w, type) per chunk in chunk order and scatters them
  // sequentially, which is the same per-cell order).
  const uint64_t s = net.step;
  auto deliver = [&](uint32_t post, uint8_t dl, uint8_t st, T wv) {
    if (net.receptor) {  // synaptic.rs:114-127: jump the receptor's conductance now
      net.rg[(size_t)receptor_of(st) * N + post] += wv;
      return;
    }
    uint32_t ts = (uint32_t)((s + std::max<uint32_t>(dl, 1)) % kSlots);
    net.ring_slot(st, ts)[post] += wv;
  };
  // the delivered weight of edge e: its weight, scaled by R*U for a
  // short-term-plastic edge (P/api/net/push.rs:83-102; each edge fires at most
  // once per step, so the push threads update disjoint edge states)
  auto tm_weight = [&](uint64_t e) -> T {
    if (net.tm.empty() || net.pt[e] == 0) return net.w[e];
    return (T)tm_spike(net.tm[net.pt[e] - 1], net.tm_r[e], net.tm_u[e], net.tm_last[e], (float)net.w[e], s);
  };
  if (g_threads > 1 && net.active.size() > 64) {
    struct Tri {
      uint32_t post;
      uint8_t d, st;
      T w;
    };
    const size_t A = net.active.size();
    const int nt = g_threads;
    const size_t chunk = std::max<size_t>((A + nt - 1) / nt, 8);
    std::vector<std::vector<Tri>> parts(nt);
    auto work = [&](int t) {
      size_t a0 = std::min(A, (size_t)t * chunk), a1 = std::min(A, a0 + chunk);
      auto &out = parts[t];
      for (size_t a = a0; a < a1; ++a) {
        uint32_t pre = net.active[a];
        for (uint64_t e = net.row_ptr[pre]; e < net.row_ptr[pre + 1]; ++e)
          out.push_back(Tri{net.col[e], net.d[e], net.st[e], tm_weight(e)});
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    for (auto &part : parts)
      for (auto &t : part) deliver(t.post, t.d, t.st, t.w);
  } else {
    for (uint32_t pre : net.active)
      for (uint64_t e = net.row_ptr[pre]; e < net.row_ptr[pre + 1]; ++e)
        deliver(net.col[e], net.d[e], net.st[e], tm_weight(e));
  }
  for (uint32_t pre : net.active) net.events += net.row_ptr[pre + 1] - net.row_ptr[pre];
  // 5b. Poisson sources (step.rs:163-185)
  for (auto &src : net.srcs) {
    if (src.p <= 0.0f || !poisson_spike(src.seed, 0, s, src.p)) continue;
    for (size_t i = 0; i < src.post.size(); ++i) {
      T w = src.w[i];
      if (src.pt[i])  // step.rs:172-177: the synapse's short-term plasticity scales the weight
        w = (T)tm_spike(net.tm[src.pt[i] - 1], src.r[i], src.u[i], src.last[i], (float)src.w[i], s);
      deliver(src.post[i], src.d[i], src.st[i], w);
    }
    net.events += src.post.size();
  }
  // Pair STDP with immediate weight updates (oracle-defined; trace order
  // from P/api/learn/brain.rs:204-222: decay then add, fused mul_add,
  // d = fast_exp(-dt/tau)).  Depression on the out-edges of every spiking
  // pre, then potentiation on the in-edges of every spiking post; each
  // update is clipped to [w_min, w_max].  The push above used the weights
  // from before this step's update.
  if (net.stdp.on) {
    const Stdp &c = net.stdp;
    const T d_pre = M<T>::fexp(-(T)c.dt / (T)c.tau_pre);
    const T d_post = M<T>::fexp(-(T)c.dt / (T)c.tau_post);
    for (size_t i = 0; i < N; ++i) {
      T add = net.spikes[i] > 0 ? (T)1 : (T)0;
      net.x_pre[i] = M<T>::fma(net.x_pre[i], d_pre, add);
      net.x_post[i] = M<T>::fma(net.x_post[i], d_post, add);
    }
    const T wmin = (T)c.w_min, wmax = (T)c.w_max, am = (T)c.a_minus, ap = (T)c.a_plus;
    for (uint32_t pre : net.active)
      for (uint64_t e = net.row_ptr[pre]; e < net.row_ptr[pre + 1]; ++e) {
        if (!net.plastic[e]) continue;
        T w0 = net.w[e];
        T w1 = std::fmin(std::fmax(w0 - am * net.x_post[net.col[e]], wmin), wmax);
        net.w[e] = w1;
        net.drift += (double)w1 - (double)w0;
      }
    for (uint32_t post : net.active)
      for (uint64_t k = net.in_ptr[post]; k < net.in_ptr[post + 1]; ++k) {
        uint32_t e = net.in_edge[k];
        uint32_t pre = net.in_pre[k];
        T w0 = net.w[e];
        T w1 = std::fmin(std::fmax(w0 + ap * net.x_pre[pre], wmin), wmax);
        net.w[e] = w1;
        net.drift += (double)w1 - (double)w0;
      }
  }
  if (net.learn.on) learn_step(net);
  net.step++;
}

template <typename T> void net_step(Net<T> &net) {
  net_step_begin(net);
  net_step_end(net);
}

// P/api/learn/brain.rs:204-286 Brain::step: traces decay and take this
// step's spikes (fused mul_add); every spike stages an event for each of its
// neuron's in-edges (+a_ltp * pre trace) then out-edges (-a_ltd * post
// trace), neurons ascending; phase A brings each touched synapse's
// eligibility from its last sync by repeated multiplication with d_e and adds
// the events in order, phase B applies one trailing decay per touched synapse.
template <typename T> void learn_step(Net<T> &net) {
  Learn &L = net.learn;
  const size_t N = net.total;
  L.t += 1;
  const uint64_t t = L.t;
  const float d_pre = fast_exp_f(-L.dt / L.tau_pre), d_post = fast_exp_f(-L.dt / L.tau_post);
  const float d_e = fast_exp_f(-L.dt / L.tau_e);
  for (size_t n = 0; n < N; ++n) {
    const float add = net.spikes[n] > 0 ? 1.0f : 0.0f;
    L.tp[n] = std::fma(L.tp[n], d_pre, add);
    L.tq[n] = std::fma(L.tq[n], d_post, add);
    if (net.spikes[n] != 0)
      for (int m = 0; m < 2; ++m) L.motor[m] += (n >= L.motor_lo[m] && n < L.motor_hi[m]) ? 1u : 0u;
  }
  L.events.clear();
  for (size_t n = 0; n < N; ++n) {
    if (net.spikes[n] == 0) continue;
    for (uint32_t k = L.in_ptr[n]; k < L.in_ptr[n + 1]; ++k) {
      const uint32_t i = L.in_edge[k];
      L.events.push_back({i, L.a_ltp * L.tp[L.pre_of[i]]});
    }
    for (uint64_t e = net.row_ptr[n]; e < net.row_ptr[n + 1]; ++e)
      L.events.push_back({(uint32_t)e, -L.a_ltd * L.tq[net.col[e]]});
  }
  for (auto &ev : L.events) {
    float &e = L.elig[ev.first];
    const uint64_t s0 = L.last[ev.first];
    if (s0 < t) {
      for (uint64_t k = 1; k < t - s0; ++k) e *= d_e;
      L.last[ev.first] = t;
    }
    e += ev.second;
  }
  for (auto &ev : L.events)
    if (L.stamp[ev.first] != t) {
      L.stamp[ev.first] = t;
      L.elig[ev.first] *= d_e;
    }
}

struct Handle {
  int precision;
  NetBase *net;
};

template <typename T> Net<T> &N_(const or_net *h) {
  return *static_cast<Net<T> *>(((Handle *)const_cast<or_net *>(h))->net);
}

#define DISPATCH(h, ...)                           \
  do {                                             \
    if (((const Handle *)(h))->precision == 0) {   \
      auto &net = N_<float>(h);                    \
      __VA_ARGS__;                                 \
    } else {                                       \
      auto &net = N_<double>(h);                   \
      __VA_ARGS__;                                 \
    }                                              \
  } while (0)

template <typename T> int pop_check(Net<T> &net, int pop, int col, bool param) {
  if (pop < 0 || (size_t)pop >= net.pops.size()) return fail("population out of range");
  auto &p = net.pops[pop];
  int lim = param ? (int)p.np : (int)p.ns;
  if (col < 0 || col >= lim) return fail("column out of range");
  return 0;
}

template <typename T> int kuramoto_rk4(uint32_t n, const float *th0, const float *om, float kf,
                                       float dtf, uint32_t steps, float *th_out, double *r_out) {
  std::vector<T> th(n), omg(n), k1(n), k2(n), k3(n), k4(n), tmp(n);
  for (uint32_t i = 0; i < n; ++i) {
    th[i] = (T)th0[i];
    omg[i] = (T)om[i];
  }
  const T K = (T)kf, dt = (T)dtf, hdt = dt * (T)0.5f, inv_n = (T)1 / (T)n;
  const T two_pi = (T)6.28318530717958647692;
  auto field = [&](const std::vector<T> &x, std::vector<T> &k) {
    double cs = 0, sn = 0;
    for (uint32_t i = 0; i < n; ++i) {
      cs += std::cos((double)x[i]);
      sn += std::sin((double)x[i]);
    }
    T C = (T)(cs / n), S = (T)(sn / n);
    for (uint32_t i = 0; i < n; ++i) k[i] = omg[i] + K * (S * std::cos(x[i]) - C * std::sin(x[i]));
  };
  (void)inv_n;
  for (uint32_t s = 0; s < steps; ++s) {
    field(th, k1);
    for (uint32_t i = 0; i < n; ++i) tmp[i] = th[i] + hdt * k1[i];
    field(tmp, k2);
    for (uint32_t i = 0; i < n; ++i) tmp[i] = th[i] + hdt * k2[i];
    field(tmp, k3);
    for (uint32_t i = 0; i < n; ++i) tmp[i] = th[i] + dt * k3[i];
    field(tmp, k4);
    const T w6 = dt / (T)6;
    for (uint32_t i = 0; i < n; ++i) {
      T x = th[i] + w6 * (((k1[i] + (T)2 * k2[i]) + (T)2 * k3[i]) + k4[i]);
      th[i] = x - two_pi * std::round(x / two_pi);  // P/kernels/mod.rs:74-77
    }
    if (r_out) {
      double cs = 0, sn = 0;
      for (uint32_t i = 0; i < n; ++i) {
        cs += std::cos((double)th[i]);
        sn += std::sin((double)th[i]);
      }
      r_out[s] = std::sqrt(cs * cs + sn * sn) / n;
    }
  }
  for (uint32_t i = 0; i < n; ++i) th_out[i] = (float)th[i];
  return 0;
}

}  // namespace

// ===========================================================================
// C API
// ===========================================================================
extern "C" {

const char *or_last_error(void) { return g_err.c_str(); }

or_net *or_net_new(int precision) {
  Handle *h = new Handle;
  h->precision = precision ? 1 : 0;
  if (h->precision == 0) h->net = new Net<float>();
  else h->net = new Net<double>();
  return (or_net *)h;
}

void or_net_free(or_net *h) {
  if (!h) return;
  delete ((Handle *)h)->net;
  delete (Handle *)h;
}

int or_set_threads(int n) {
  g_threads = n < 1 ? 1 : n;
  return g_threads;
}

// P/api/net/network/core.rs:124-155 add_population; capacity = ceil(n/8)*8
int or_pop_add(or_net *h, int model, uint32_t n) {
  int np = n_params_of(model), ns = n_state_of(model);
  if (np < 0) return fail("unknown model");
  int id = -1;
  DISPATCH(h, {
    if (net.built) return fail("Cannot add populations after build()");
    if (net.total + n > 0xFFFFFFFFull) return fail("Network: total neuron count exceeds u32::MAX");
    Pop<std::remove_reference_t<decltype(net.w[0])>> p;
    p.model = model;
    p.n = n;
    p.cap = (n + 7) / 8 * 8;
    p.np = np;
    p.ns = ns;
    p.params.assign((size_t)p.cap * np, 0);
    p.state.assign((size_t)p.cap * ns, 0);
    net.pops.push_back(std::move(p));
    net.total += n;
    net.offsets.push_back((uint32_t)net.total);
    id = (int)net.pops.size() - 1;
  });
  return id;
}

// A population simulated by another rank of a split network: no state or
// parameters here, its spikes of each step set by or_set_external_spikes
// between or_step_begin and or_step_end.
int or_pop_add_external(or_net *h, uint32_t n) {
  int id = -1;
  DISPATCH(h, {
    if (net.built) return fail("Cannot add populations after build()");
    if (net.total + n > 0xFFFFFFFFull) return fail("Network: total neuron count exceeds u32::MAX");
    Pop<std::remove_reference_t<decltype(net.w[0])>> p;
    p.model = 0;
    p.n = n;
    p.cap = (n + 7) / 8 * 8;
    p.np = p.ns = 0;
    net.pops.push_back(std::move(p));
    net.total += n;
    net.offsets.push_back((uint32_t)net.total);
    id = (int)net.pops.size() - 1;
  });
  return id;
}

int or_pop_fill_param(or_net *h, int pop, int col, double v) {
  DISPATCH(h, {
    if (pop_check(net, pop, col, true)) return -1;
    auto &p = net.pops[pop];
    for (uint32_t i = 0; i < p.n; ++i) p.params[(size_t)col * p.cap + i] = (decltype(p.params[0] + 0))(float)v;
  });
  return 0;
}
int or_pop_fill_state(or_net *h, int pop, int col, double v) {
  DISPATCH(h, {
    if (pop_check(net, pop, col, false)) return -1;
    auto &p = net.pops[pop];
    for (uint32_t i = 0; i < p.n; ++i) p.state[(size_t)col * p.cap + i] = (decltype(p.state[0] + 0))(float)v;
  });
  return 0;
}
int or_pop_set_param(or_net *h, int pop, int col, const float *v, uint32_t n) {
  DISPATCH(h, {
    if (pop_check(net, pop, col, true)) return -1;
    auto &p = net.pops[pop];
    if (n != p.n) return fail("length mismatch");
    for (uint32_t i = 0; i < p.n; ++i) p.params[(size_t)col * p.cap + i] = v[i];
  });
  return 0;
}
int or_pop_set_state(or_net *h, int pop, int col, const float *v, uint32_t n) {
  DISPATCH(h, {
    if (pop_check(net, pop, col, false)) return -1;
    auto &p = net.pops[pop];
    if (n != p.n) return fail("length mismatch");
    for (uint32_t i = 0; i < p.n; ++i) p.state[(size_t)col * p.cap + i] = v[i];
  });
  return 0;
}
int or_pop_get_state(or_net *h, int pop, int col, float *out, uint32_t n) {
  DISPATCH(h, {
    if (pop_check(net, pop, col, false)) return -1;
    auto &p = net.pops[pop];
    if (n != p.n) return fail("length mismatch");
    for (uint32_t i = 0; i < p.n; ++i) out[i] = (float)p.state[(size_t)col * p.cap + i];
  });
  return 0;
}
int or_pop_get_state_f64(or_net *h, int pop, int col, double *out, uint32_t n) {
  DISPATCH(h, {
    if (pop_check(net, pop, col, false)) return -1;
    auto &p = net.pops[pop];
    if (n != p.n) return fail("length mismatch");
    for (uint32_t i = 0; i < p.n; ++i) out[i] = (double)p.state[(size_t)col * p.cap + i];
  });
  return 0;
}
int or_pop_get_param(or_net *h, int pop, int col, float *out, uint32_t n) {
  DISPATCH(h, {
    if (pop_check(net, pop, col, true)) return -1;
    auto &p = net.pops[pop];
    if (n != p.n) return fail("length mismatch");
    for (uint32_t i = 0; i < p.n; ++i) out[i] = (float)p.params[(size_t)col * p.cap + i];
  });
  return 0;
}

// P/api/net/network/core.rs:166-249 connect / connect_inner
int or_connect(or_net *h, int from, const uint32_t *fi, int to, const uint32_t *ti, const float *w,
               const uint8_t *dl, const uint8_t *st, const uint8_t *pt, uint64_t n, uint32_t flags) {
  DISPATCH(h, {
    if (net.built) return fail("Cannot connect after build()");
    if (from < 0 || (size_t)from >= net.pops.size()) return fail("from population out of range");
    if (to < 0 || (size_t)to >= net.pops.size()) return fail("to population out of range");
    if (net.pops[to].model == 0) return fail("no synapses onto an external population");
    const uint32_t fo = net.offsets[from], fc = net.offsets[from + 1] - fo;
    const uint32_t tof = net.offsets[to], tc = net.offsets[to + 1] - tof;
    for (uint64_t i = 0; i < n; ++i) {
      if (fi[i] >= fc) return fail("from index out of bounds");
      if (ti[i] >= tc) return fail("to index out of bounds");
      if (!std::isfinite(w[i])) return fail("Network::connect: weight must be finite");
      if (dl[i] >= kSlots) return fail("delay >= MAX_DELAY_SLOTS");
      uint8_t s = st ? st[i] : 0;
      const uint8_t p = pt ? pt[i] : 0;
      if (p > net.tm.size()) return fail("Network::build: plast_type exceeds registered plasticity profiles");
      net.edges.push_back(EdgeIn{fo + fi[i], tof + ti[i], w[i], dl[i], s, (uint8_t)(flags & 1), p});
    }
  });
  return 0;
}

// P/api/net/network/core.rs:586-623 register_plasticity, validation of
// P/api/net/synapse.rs:268-292; a_rec = exp(-dt/tau_rec) in f32 on the host
int or_register_plasticity(or_net *h, float u0, float tau_rec, int facilitation, float tau_fac, float dt) {
  int id = -1;
  if (!(dt > 0) || !std::isfinite(dt)) return fail("register_plasticity: dt must be finite and > 0");
  if (!std::isfinite(u0) || u0 <= 0.0f || u0 > 1.0f) return fail("init_release_prob must be in (0, 1]");
  if (!std::isfinite(tau_rec) || tau_rec <= 0.0f) return fail("tau_rec must be finite and > 0");
  if (facilitation && (!std::isfinite(tau_fac) || tau_fac <= 0.0f)) return fail("tau_fac must be finite and > 0");
  DISPATCH(h, {
    if (net.built) return fail("register_plasticity must be called before build()");
    if (net.tm.size() >= 255) return fail("profile id overflow");
    net.tm.push_back(TmProf{u0, std::exp(-dt / tau_rec), facilitation ? std::exp(-dt / tau_fac) : 0.0f,
                            facilitation != 0});
    id = (int)net.tm.size();
  });
  return id;
}

// tm_spike on one synapse over a spike sequence (the reference's NEURON
// goldens, P/api/net/push.rs:646-695): out[k] = delivered weight of a spike
// of weight w at steps[k]
int or_tm_sequence(float u0, float a_rec, float a_fac, int facilitation, float w, const uint64_t *steps,
                   uint32_t n, float *out) {
  TmProf p{u0, a_rec, a_fac, facilitation != 0};
  float r = 1.0f, u = u0;
  uint32_t last = 0;
  for (uint32_t k = 0; k < n; ++k) out[k] = tm_spike(p, r, u, last, w, steps[k]);
  return 0;
}

// Learning over the built network's synapses (Brain::new, brain.rs:106-141):
// in-edges per post in CSR index order, traces and eligibility zero.
int or_learn_enable(or_net *h, float dt, float tau_pre, float tau_post, float tau_e, float a_ltp, float a_ltd,
                    float lr, float w_min, float w_max) {
  DISPATCH(h, {
    if (!net.built) return fail("learning needs a built network");
    Learn &L = net.learn;
    L = Learn{};
    L.on = true;
    L.dt = dt, L.tau_pre = tau_pre, L.tau_post = tau_post, L.tau_e = tau_e;
    L.a_ltp = a_ltp, L.a_ltd = a_ltd, L.lr = lr, L.w_min = w_min, L.w_max = w_max;
    const size_t N = net.total, E = net.col.size();
    L.tp.assign(N, 0.0f);
    L.tq.assign(N, 0.0f);
    L.elig.assign(E, 0.0f);
    L.last.assign(E, 0);
    L.stamp.assign(E, 0);
    L.pre_of.assign(E, 0);
    std::vector<uint64_t> cnt(N + 1, 0);
    for (uint64_t pre = 0; pre < N; ++pre)
      for (uint64_t e = net.row_ptr[pre]; e < net.row_ptr[pre + 1]; ++e) {
        L.pre_of[e] = (uint32_t)pre;
        cnt[net.col[e]]++;
      }
    L.in_ptr.assign(N + 1, 0);
    for (size_t i = 0; i < N; ++i) L.in_ptr[i + 1] = L.in_ptr[i] + (uint32_t)cnt[i];
    L.in_edge.assign(E, 0);
    std::vector<uint32_t> cur(L.in_ptr.begin(), L.in_ptr.end() - 1);
    for (uint64_t e = 0; e < E; ++e) L.in_edge[cur[net.col[e]]++] = (uint32_t)e;
  });
  return 0;
}

// brain.rs:288-341 fold_eligibility + reward_dopamine: every eligibility is
// brought to now by repeated multiplication, then w += lr*dopamine*e clamped to
// [w_min, cap] (cap: w_max unless w_cap is finite); zero deltas leave w alone.
// Reward of the synapses [lo, hi) only: in a pool of independent networks
// (populations without synapses between them) one network's synapses are
// one CSR range, and its reward is then exactly its own Brain's.
int or_learn_reward_range(or_net *h, uint64_t lo, uint64_t hi, float dopamine, float gate, float w_cap) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    if (lo > hi || hi > L.elig.size()) return fail("synapse range out of bounds");
    const float w_max = std::isfinite(w_cap) ? w_cap : L.w_max;
    if (!(L.w_min <= w_max)) return fail("weight ceiling below the floor");
    // reward_gated: dopamine * gate.clamp(0, 1) (brain.rs:405-409)
    const float g = gate < 0.0f ? 0.0f : (gate > 1.0f ? 1.0f : gate);
    const float dop = dopamine * g;
    const float d_e = fast_exp_f(-L.dt / L.tau_e);
    for (size_t i = lo; i < hi; ++i) {
      const uint64_t s0 = L.last[i];
      if (s0 < L.t && L.elig[i] != 0.0f) {
        for (uint64_t k = 0; k < L.t - s0; ++k) L.elig[i] *= d_e;
        L.last[i] = L.t;
      } else if (s0 < L.t) {
        L.last[i] = L.t;
      }
    }
    const float lr_dopa = L.lr * dop;
    for (size_t i = lo; i < hi; ++i) {
      const float delta = lr_dopa * L.elig[i];
      if (delta == 0.0f) continue;
      const float w = (float)net.w[i] + delta;
      net.w[i] = (std::decay_t<decltype(net.w[i])>)(w < L.w_min ? L.w_min : (w > w_max ? w_max : w));
    }
  });
  return 0;
}

int or_learn_reward(or_net *h, float dopamine, float gate, float w_cap) {
  uint64_t E = 0;
  DISPATCH(h, { E = net.learn.elig.size(); });
  return or_learn_reward_range(h, 0, E, dopamine, gate, w_cap);
}

// brain.rs:271-280 clear_eligibility: zero, synced to now (of [lo, hi))
int or_learn_clear_range(or_net *h, uint64_t lo, uint64_t hi) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    if (lo > hi || hi > L.elig.size()) return fail("synapse range out of bounds");
    std::fill(L.elig.begin() + lo, L.elig.begin() + hi, 0.0f);
    std::fill(L.last.begin() + lo, L.last.begin() + hi, L.t);
  });
  return 0;
}

int or_learn_clear(or_net *h) {
  uint64_t E = 0;
  DISPATCH(h, { E = net.learn.elig.size(); });
  return or_learn_clear_range(h, 0, E);
}

// the CSR synapse range of a population's rows
int or_pop_synapse_range(or_net *h, int pop, uint64_t *lo, uint64_t *hi) {
  DISPATCH(h, {
    if (!net.built) return fail("not built");
    if (pop < 0 || (size_t)pop >= net.pops.size()) return fail("population out of range");
    *lo = net.row_ptr[net.offsets[pop]];
    *hi = net.row_ptr[net.offsets[pop + 1]];
  });
  return 0;
}

// brain.rs:282-289 restrict_eligibility: keep[i] == 0 zeroes synapse i
int or_learn_restrict(or_net *h, const uint8_t *keep, uint64_t n) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    for (uint64_t i = 0; i < n && i < L.elig.size(); ++i)
      if (!keep[i]) L.elig[i] = 0.0f;
  });
  return 0;
}

// brain.rs:160-170 set_eligibility: values replaced, sync steps kept
int or_learn_set_eligibility(or_net *h, const float *elig, uint64_t n) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    if (n != L.elig.size()) return fail("eligibility length differs from the synapse count");
    std::copy(elig, elig + n, L.elig.begin());
  });
  return 0;
}

int or_learn_motor(or_net *h, uint64_t lo0, uint64_t hi0, uint64_t lo1, uint64_t hi1) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    L.motor_lo[0] = lo0, L.motor_hi[0] = hi0, L.motor_lo[1] = lo1, L.motor_hi[1] = hi1;
  });
  return 0;
}

int or_learn_motor_read(or_net *h, uint32_t *out) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    out[0] = L.motor[0], out[1] = L.motor[1];
  });
  return 0;
}

// brain.rs:343-356 snapshot / recall: w += alpha * (snapshot - w)
int or_learn_snapshot(or_net *h) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    L.baked.assign(net.w.begin(), net.w.end());
  });
  return 0;
}

int or_learn_recall(or_net *h, float alpha) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    for (size_t i = 0; i < L.baked.size() && i < net.w.size(); ++i) {
      const float w = (float)net.w[i];
      net.w[i] = (std::decay_t<decltype(net.w[i])>)(w + alpha * (L.baked[i] - w));
    }
  });
  return 0;
}

int or_learn_read(or_net *h, float *elig, float *tp, float *tq, uint64_t *t) {
  DISPATCH(h, {
    Learn &L = net.learn;
    if (!L.on) return fail("learning is not enabled");
    if (elig) std::copy(L.elig.begin(), L.elig.end(), elig);
    if (tp) std::copy(L.tp.begin(), L.tp.end(), tp);
    if (tq) std::copy(L.tq.begin(), L.tq.end(), tq);
    if (t) *t = L.t;
  });
  return 0;
}

// P/api/net/network/core.rs:564-584 register_kinetics for every waveform
// kind, validation of P/api/net/synapse.rs:95-158, constants of
// step.rs:249-297.  p: ExpOne {tau_decay}, ExpTwo {tau_rise, tau_decay},
// Alpha {tau}, ExpThree {tau_rise, tau_decay1, tau_decay2, gbase1, gbase2}.
int or_register_kinetics(or_net *h, int kind, const float *p, float erev, float dt) {
  int id = -1;
  auto pos = [](float x) { return std::isfinite(x) && x > 0.0f; };
  if (!std::isfinite(erev)) return fail("erev must be finite");
  if (!(dt > 0) || !std::isfinite(dt)) return fail("register_kinetics: dt must be finite and > 0");
  Kin k{kind, erev, {}};
  if (kind == 0) {
    if (!pos(p[0])) return fail("tau_decay must be finite and > 0");
    k.c[0] = std::exp(-dt / p[0]);
  } else if (kind == 1) {
    if (!pos(p[1])) return fail("tau_decay must be finite and > 0");
    if (!pos(p[0])) return fail("tau_rise must be finite and > 0");
    if (p[0] >= p[1]) return fail("tau_rise must be < tau_decay");
    k.c[0] = std::exp(-dt / p[0]);
    k.c[1] = std::exp(-dt / p[1]);
    k.c[2] = waveform_factor(p[0], p[1]);
  } else if (kind == 2) {
    if (!pos(p[0])) return fail("tau must be finite and > 0");
    const float r = std::exp(-dt / p[0]);
    k.c[0] = r;
    k.c[1] = 2.7182817f * (dt / p[0]) * r;  // std::f32::consts::E
  } else if (kind == 3) {
    const float tr = p[0], td1 = p[1], td2 = p[2], g1 = p[3], g2 = p[4];
    if (!pos(tr)) return fail("tau_rise must be finite and > 0");
    if (!std::isfinite(td1) || td1 <= tr) return fail("tau_decay1 must be finite and > tau_rise");
    if (!std::isfinite(td2) || td2 <= tr) return fail("tau_decay2 must be finite and > tau_rise");
    if (!std::isfinite(g1) || g1 < 0.0f || !std::isfinite(g2) || g2 < 0.0f) return fail("gbase must be finite and >= 0");
    if (g1 + g2 <= 0.0f) return fail("gbase1 + gbase2 must be > 0");
    const float wf1 = waveform_factor(tr, td1), wf2 = waveform_factor(tr, td2);
    k.c[0] = std::exp(-dt / tr);
    k.c[1] = std::exp(-dt / td1);
    k.c[2] = std::exp(-dt / td2);
    k.c[3] = wf1;
    k.c[4] = wf2;
    k.c[5] = (g1 * wf1 + g2 * wf2) / (g1 + g2);
    k.c[6] = g1;
    k.c[7] = g2;
  } else {
    return fail("unknown kinetics kind");
  }
  DISPATCH(h, {
    if (net.built) return fail("register_kinetics must be called before build()");
    if (net.kin.size() >= 255) return fail("profile id overflow");
    net.kin.push_back(k);
    id = (int)net.kin.size();
  });
  return id;
}

// P/api/net/network/core.rs:564-584 register_kinetics (ExpOne profile,
// a_decay = exp(-dt/tau) in f32, step.rs:252-254)
int or_register_expone(or_net *h, float tau_decay, float erev, float dt) {
  int id = -1;
  if (!(tau_decay > 0) || !std::isfinite(tau_decay)) return fail("tau_decay must be finite and > 0");
  if (!(dt > 0) || !std::isfinite(dt)) return fail("register_kinetics: dt must be finite and > 0");
  DISPATCH(h, {
    if (net.built) return fail("register_kinetics must be called before build()");
    if (net.kin.size() >= 255) return fail("profile id overflow");
    Kin k{0, erev, {std::exp(-dt / tau_decay)}};
    net.kin.push_back(k);
    id = (int)net.kin.size();
  });
  return id;
}

// SynapticBrain::from_sparse_graph(graph, receptor_types, dt)
// (pillars-connectome/src/synaptic.rs:53-63) on this network: the edges'
// syn_types become receptor codes (code >= 7 is AMPA), delays are ignored
// (a spike jumps its targets' conductances at once), DecayFactors::new(dt).
int or_set_receptor_kinetics(or_net *h, float dt) {
  if (!(dt > 0) || !std::isfinite(dt)) return fail("receptor kinetics: dt must be finite and > 0");
  DISPATCH(h, {
    if (net.built) return fail("receptor kinetics must be set before build()");
    net.receptor = true;
    net.rec_dt = dt;
  });
  return 0;
}

// SynapticBrain::kinetics / set_kinetics (synaptic.rs:72-80): the seven
// conductance arrays, [7][total] in receptor-code order.
int or_receptor_read(or_net *h, float *g) {
  DISPATCH(h, {
    if (!net.built || !net.receptor) return fail("receptor kinetics are not on");
    for (size_t k = 0; k < net.rg.size(); ++k) g[k] = (float)net.rg[k];
  });
  return 0;
}

int or_receptor_factors(float dt, float *f) {
  if (!(dt > 0) || !std::isfinite(dt)) return fail("receptor kinetics: dt must be finite and > 0");
  receptor_factors(dt, f);
  return 0;
}

// I_out[i] = sum over receptors of g_eff (E_rev - v[i]) for n neurons with
// conductances g[r * n + i] (SynapticKinetics::compute_currents into a zeroed
// output).
int or_receptor_currents(uint32_t n, const float *g, const float *v, float *i_out) {
  for (uint32_t i = 0; i < n; ++i) {
    float gi[kReceptors];
    for (int r = 0; r < kReceptors; ++r) gi[r] = g[(size_t)r * n + i];
    i_out[i] = receptor_current(gi, v[i]);
  }
  return 0;
}

float or_nmda_mg_block(float v) { return nmda_mg_block(v); }

int or_receptor_write(or_net *h, const float *g) {
  DISPATCH(h, {
    if (!net.built || !net.receptor) return fail("receptor kinetics are not on");
    for (size_t k = 0; k < net.rg.size(); ++k) net.rg[k] = g[k];
  });
  return 0;
}

// P/api/net/network/core.rs:288-312
int or_poisson_add(or_net *h, float rate_hz, float dt_ms, uint32_t seed) {
  if (!std::isfinite(rate_hz) || rate_hz < 0) return fail("add_poisson_source: rate_hz must be finite and >= 0");
  if (!std::isfinite(dt_ms) || !(dt_ms > 0)) return fail("add_poisson_source: dt_ms must be finite and > 0");
  int id = -1;
  DISPATCH(h, {
    if (net.built) return fail("add_poisson_source must be called before build()");
    float p = rate_hz * dt_ms / 1000.0f;
    p = std::fmin(std::fmax(p, 0.0f), 1.0f);
    Src<std::remove_reference_t<decltype(net.w[0])>> s;
    s.p = p;
    s.seed = seed;
    net.srcs.push_back(std::move(s));
    id = (int)net.srcs.size() - 1;
  });
  return id;
}

int or_poisson_add_many(or_net *h, uint32_t n, float rate_hz, float dt_ms, uint32_t seed0) {
  int first = -1;
  for (uint32_t i = 0; i < n; ++i) {
    int id = or_poisson_add(h, rate_hz, dt_ms, seed0 + i);
    if (id < 0) return id;
    if (i == 0) first = id;
  }
  return first;
}

// P/api/net/network/core.rs:323-381
// Network::connect_poisson_source (core.rs:323-380), with the synapses'
// plasticity profiles (plast_types; NULL = none): R = 1, U = U0 of the profile
// registered when the synapse is connected, last = 0.
int or_poisson_connect_plastic(or_net *h, int src, int to, const uint32_t *posts, const float *w,
                               const uint8_t *dl, const uint8_t *st, const uint8_t *pt, uint64_t n) {
  DISPATCH(h, {
    if (net.built) return fail("Cannot connect after build()");
    if (src < 0 || (size_t)src >= net.srcs.size()) return fail("poisson source out of range");
    if (to < 0 || (size_t)to >= net.pops.size()) return fail("to population out of range");
    if (net.pops[to].model == 0) return fail("no synapses onto an external population");
    const uint32_t tof = net.offsets[to], tc = net.offsets[to + 1] - tof;
    auto &s = net.srcs[src];
    for (uint64_t i = 0; i < n; ++i) {
      if (posts[i] >= tc) return fail("post index out of bounds");
      if (!std::isfinite(w[i])) return fail("connect_poisson_source: weight must be finite");
      if (dl[i] >= kSlots) return fail("connect_poisson_source: delay >= MAX_DELAY_SLOTS");
      const uint8_t p = pt ? pt[i] : 0;
      if (p > net.tm.size()) return fail("plasticity profile out of range");
      s.post.push_back(tof + posts[i]);
      s.w.push_back(w[i]);
      s.d.push_back(dl[i]);
      s.st.push_back(st ? st[i] : 0);
      s.pt.push_back(p);
      s.r.push_back(1.0f);
      s.u.push_back(p ? net.tm[p - 1].u0 : 0.0f);
      s.last.push_back(0u);
    }
  });
  return 0;
}

int or_poisson_connect(or_net *h, int src, int to, const uint32_t *posts, const float *w,
                       const uint8_t *dl, const uint8_t *st, uint64_t n) {
  return or_poisson_connect_plastic(h, src, to, posts, w, dl, st, nullptr, n);
}

int or_poisson_connect_one_to_one(or_net *h, int first, uint32_t n, int to, float w, uint8_t dl) {
  for (uint32_t i = 0; i < n; ++i) {
    uint8_t st = 0;
    int rc = or_poisson_connect(h, first + (int)i, to, &i, &w, &dl, &st, 1);
    if (rc < 0) return rc;
  }
  return 0;
}

int or_stdp_config(or_net *h, float dt, float tau_pre, float tau_post, float a_plus, float a_minus,
                   float w_min, float w_max) {
  DISPATCH(h, {
    if (net.built) return fail("stdp must be configured before build()");
    net.stdp = Stdp{true, dt, tau_pre, tau_post, a_plus, a_minus, w_min, w_max};
  });
  return 0;
}

static inline uint64_t splitmix64_h(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// connect(fixed in-degree projection, same generator as the product's
// sg_connect_fixed_indegree: edge t = (post j, draw q) = j*k_in + q) followed
// by build(), writing the stable-sorted CSR directly (no triplet list), in
// parallel over post ranges with per-thread row offsets so that every row
// keeps (post, draw) order.  Only for a network with no other synapses.
int or_build_fixed_indegree(or_net *h, int from, int to, uint32_t k_in, uint64_t seed, uint32_t n_exc,
                            float w_exc, float w_inh, uint32_t d_min, uint32_t d_max) {
  DISPATCH(h, {
    if (net.built) return fail("Network::build() called twice");
    if (!net.edges.empty()) return fail("fixed in-degree build needs a network without other edges");
    if (from < 0 || (size_t)from >= net.pops.size() || to < 0 || (size_t)to >= net.pops.size())
      return fail("population out of range");
    if (d_min > d_max || d_max >= kSlots) return fail("delay range invalid");
    const uint32_t fo = net.offsets[from], nf = net.offsets[from + 1] - fo;
    const uint32_t tof = net.offsets[to], nt = net.offsets[to + 1] - tof;
    const uint64_t N = net.total, E = (uint64_t)nt * k_in;
    if (E > 0xFFFFFFFFull) return fail("SparseGraph: too many synapses for a u32 CSR row_ptr");
    const uint32_t span = d_max - d_min + 1;
    const int T = std::max(1, g_threads);
    auto edge = [&](uint64_t t, uint32_t &pre, uint32_t &dl) {
      const uint64_t hh = splitmix64_h(seed ^ (t * 0x9E3779B97F4A7C15ull));
      pre = (uint32_t)(((hh >> 32) * (uint64_t)nf) >> 32);
      dl = d_min + (uint32_t)((hh & 0xffffffffull) % span);
    };
    std::vector<std::vector<uint32_t>> cnt(T, std::vector<uint32_t>(N, 0));
    auto range = [&](int t, uint32_t &j0, uint32_t &j1) {
      j0 = (uint32_t)((uint64_t)nt * t / T);
      j1 = (uint32_t)((uint64_t)nt * (t + 1) / T);
    };
    auto count = [&](int t) {
      uint32_t j0, j1;
      range(t, j0, j1);
      for (uint64_t e = (uint64_t)j0 * k_in; e < (uint64_t)j1 * k_in; ++e) {
        uint32_t pre, dl;
        edge(e, pre, dl);
        cnt[t][fo + pre]++;
      }
    };
    {
      std::vector<std::thread> pool;
      for (int t = 1; t < T; ++t) pool.emplace_back(count, t);
      count(0);
      for (auto &th : pool) th.join();
    }
    net.row_ptr.assign(N + 1, 0);
    uint64_t cum = 0;
    for (uint64_t i = 0; i < N; ++i) {
      net.row_ptr[i] = (uint32_t)cum;
      for (int t = 0; t < T; ++t) {
        const uint32_t c = cnt[t][i];
        cnt[t][i] = (uint32_t)cum;  // becomes the thread's write cursor
        cum += c;
      }
    }
    net.row_ptr[N] = (uint32_t)cum;
    using TT = std::remove_reference_t<decltype(net.w[0])>;
    net.col.assign(E, 0);
    net.w.assign(E, (TT)0);
    net.d.assign(E, 0);
    net.st.assign(E, 0);
    net.plastic.assign(E, 0);
    auto fill = [&](int t) {
      uint32_t j0, j1;
      range(t, j0, j1);
      for (uint64_t e = (uint64_t)j0 * k_in; e < (uint64_t)j1 * k_in; ++e) {
        uint32_t pre, dl;
        edge(e, pre, dl);
        const uint64_t pos = cnt[t][fo + pre]++;
        net.col[pos] = tof + (uint32_t)(e / k_in);
        net.w[pos] = (TT)(pre < n_exc ? w_exc : w_inh);
        net.d[pos] = (uint8_t)dl;
      }
    };
    {
      std::vector<std::thread> pool;
      for (int t = 1; t < T; ++t) pool.emplace_back(fill, t);
      fill(0);
      for (auto &th : pool) th.join();
    }
    for (auto &sr : net.srcs)
      for (auto st : sr.st)
        if (st > net.kin.size()) return fail("Network::build: Poisson-source syn_type exceeds registered kinetics");
    alloc_runtime(net);
  });
  return 0;
}

// P/api/net/network/build.rs:18-109
int or_build(or_net *h) {
  DISPATCH(h, {
    if (net.built) return fail("Network::build() called twice");
    if (net.receptor) {
      if (!net.kin.empty() || !net.srcs.empty() || !net.tm.empty() || net.stdp.on)
        return fail("receptor kinetics: no kinetic profiles, Poisson sources, short-term or pair-STDP plasticity");
      for (auto &e : net.edges)
        if (e.flags & 1) return fail("receptor kinetics: no pair-STDP synapses");
    } else {
      for (auto &e : net.edges)
        if (e.st > net.kin.size()) return fail("Network::build: syn_type exceeds registered kinetics");
    }
    for (auto &s : net.srcs)
      for (auto st : s.st)
        if (st > net.kin.size()) return fail("Network::build: Poisson-source syn_type exceeds registered kinetics");
    if (build_csr(net)) return -1;
    alloc_runtime(net);
  });
  return 0;
}

// P/api/net/graph.rs:217-275 from_csr (all edges static, not plastic)
int or_build_from_csr(or_net *h, const uint32_t *row_ptr, const uint32_t *col, const float *w,
                      const uint8_t *dl) {
  DISPATCH(h, {
    if (net.built) return fail("Network::build() called twice");
    if (!net.edges.empty()) return fail("from_csr: edges were already added");
    const uint64_t N = net.total;
    if (row_ptr[0] != 0) return fail("CSR row_ptr must start at 0");
    for (uint64_t i = 0; i < N; ++i)
      if (row_ptr[i] > row_ptr[i + 1]) return fail("CSR row_ptr must be monotonically non-decreasing");
    const uint64_t E = row_ptr[N];
    net.row_ptr.assign(row_ptr, row_ptr + N + 1);
    net.col.assign(col, col + E);
    net.w.resize(E);
    for (uint64_t e = 0; e < E; ++e) {
      if (col[e] >= N) return fail("col index out of range");
      if (!std::isfinite(w[e])) return fail("weight must be finite");
      if (dl[e] >= kSlots) return fail("delay >= MAX_DELAY_SLOTS");
      net.w[e] = w[e];
    }
    net.d.assign(dl, dl + E);
    net.st.assign(E, 0);
    net.plastic.assign(E, 0);
    alloc_runtime(net);
  });
  return 0;
}

// P/api/net/network/build.rs:243-275 inject_current (same-step slot)
int or_inject(or_net *h, int pop, const uint32_t *idx, const float *v, uint64_t n) {
  DISPATCH(h, {
    if (!net.built) return fail("inject_current() called before build()");
    if (pop < 0 || (size_t)pop >= net.pops.size()) return fail("inject_current: population out of range");
    if (net.pops[pop].model == 0) return fail("inject_current: external population");
    const uint32_t start = net.offsets[pop], count = net.offsets[pop + 1] - start;
    for (uint64_t i = 0; i < n; ++i) {
      if (idx[i] >= count) return fail("inject_current: neuron index out of bounds");
      if (!std::isfinite(v[i])) return fail("inject_current: value must be finite");
    }
    auto *s = net.ring_slot(0, (uint32_t)(net.step % kSlots));
    for (uint64_t i = 0; i < n; ++i) s[start + idx[i]] += v[i];
  });
  return 0;
}

int or_step(or_net *h, uint32_t n_steps, uint8_t *raster) {
  DISPATCH(h, {
    if (!net.built) return fail("Network::step() called before build()");
    net.learn.motor[0] = net.learn.motor[1] = 0;
    for (uint32_t k = 0; k < n_steps; ++k) {
      net_step(net);
      if (raster)
        for (uint64_t i = 0; i < net.total; ++i) raster[(size_t)k * net.total + i] = (uint8_t)net.spikes[i];
    }
  });
  return 0;
}

int or_step_begin(or_net *h) {
  DISPATCH(h, {
    if (!net.built) return fail("Network::step() called before build()");
    net.learn.motor[0] = net.learn.motor[1] = 0;
    net_step_begin(net);
  });
  return 0;
}

int or_set_external_spikes(or_net *h, int pop, const int32_t *s, uint32_t n) {
  DISPATCH(h, {
    if (pop < 0 || (size_t)pop >= net.pops.size()) return fail("population out of range");
    if (net.pops[pop].model != 0) return fail("not an external population");
    if (n != net.pops[pop].n) return fail("length mismatch");
    for (uint32_t i = 0; i < n; ++i) net.spikes[net.offsets[pop] + i] = s[i] != 0 ? 1 : 0;
  });
  return 0;
}

int or_step_end(or_net *h) {
  DISPATCH(h, {
    if (!net.built) return fail("Network::step() called before build()");
    net_step_end(net);
  });
  return 0;
}

int or_spikes(or_net *h, int pop, int32_t *out, uint32_t n) {
  DISPATCH(h, {
    if (pop < 0 || (size_t)pop >= net.pops.size()) return fail("population out of range");
    uint32_t s = net.offsets[pop], c = net.offsets[pop + 1] - s;
    if (n != c) return fail("length mismatch");
    if (!net.built) {
      std::memset(out, 0, n * 4);
      return 0;
    }
    std::memcpy(out, &net.spikes[s], (size_t)c * 4);
  });
  return 0;
}

uint64_t or_step_counter(const or_net *h) {
  uint64_t r = 0;
  DISPATCH(h, { r = net.step; });
  return r;
}
uint64_t or_total_neurons(const or_net *h) {
  uint64_t r = 0;
  DISPATCH(h, { r = net.total; });
  return r;
}
uint64_t or_num_synapses(const or_net *h) {
  uint64_t r = 0;
  DISPATCH(h, { r = net.built ? net.col.size() : net.edges.size(); });
  return r;
}
uint64_t or_events(const or_net *h) {
  uint64_t r = 0;
  DISPATCH(h, { r = net.events; });
  return r;
}

int or_ring_read(or_net *h, int ring, float *out) {
  DISPATCH(h, {
    if (!net.built) return fail("not built");
    if (ring < 0 || (size_t)ring > net.kin.size()) return fail("ring out of range");
    const size_t cnt = (size_t)kSlots * net.total;
    const auto *src = &net.ring[(size_t)ring * cnt];
    for (size_t i = 0; i < cnt; ++i) out[i] = (float)src[i];
  });
  return 0;
}

int or_graph_read(or_net *h, uint32_t *row_ptr, uint32_t *col, float *w, uint8_t *dl) {
  DISPATCH(h, {
    if (!net.built) return fail("not built");
    std::memcpy(row_ptr, net.row_ptr.data(), net.row_ptr.size() * 4);
    std::memcpy(col, net.col.data(), net.col.size() * 4);
    for (size_t i = 0; i < net.w.size(); ++i) w[i] = (float)net.w[i];
    std::memcpy(dl, net.d.data(), net.d.size());
  });
  return 0;
}

int or_weights_read(or_net *h, float *w) {
  DISPATCH(h, {
    if (!net.built) return fail("not built");
    for (size_t i = 0; i < net.w.size(); ++i) w[i] = (float)net.w[i];
  });
  return 0;
}

// Restore CSR weights (a checkpoint's values section) into the built network.
int or_weights_write(or_net *h, const float *w, uint64_t n) {
  DISPATCH(h, {
    if (!net.built) return fail("not built");
    if (n != net.w.size()) return fail("weight count differs from the synapse count");
    for (size_t i = 0; i < net.w.size(); ++i) net.w[i] = (std::decay_t<decltype(net.w[i])>)w[i];
  });
  return 0;
}

double or_stdp_drift(const or_net *h) {
  double r = 0;
  DISPATCH(h, { r = net.drift; });
  return r;
}

int or_traces_read(or_net *h, float *x_pre, float *x_post) {
  DISPATCH(h, {
    if (!net.stdp.on || !net.built) return fail("stdp not enabled");
    for (size_t i = 0; i < net.total; ++i) {
      x_pre[i] = (float)net.x_pre[i];
      x_post[i] = (float)net.x_post[i];
    }
  });
  return 0;
}

float or_fast_exp(float x) { return fast_exp_f(x); }
float or_sg_expf(float x) { return sg_expf(x); }
float or_sg_logf(float x) { return sg_logf(x); }
int or_poisson_spike(uint32_t seed, uint32_t stream, uint64_t step, float p) {
  return poisson_spike(seed, stream, step, p) ? 1 : 0;
}
// P/api/net/push.rs:126-173 push_spikes on plain arrays (static ring)
int or_push_spikes(const uint32_t *row_ptr, const uint32_t *col, const float *w, const uint8_t *dl,
                   uint32_t n_neurons, const uint32_t *active, uint32_t n_active, uint64_t step,
                   float *ring) {
  for (uint32_t a = 0; a < n_active; ++a) {
    const uint32_t pre = active[a];
    if (pre >= n_neurons) return fail("push_spikes: active index out of range");
    for (uint32_t e = row_ptr[pre]; e < row_ptr[pre + 1]; ++e) {
      const uint32_t post = col[e];
      if (post >= n_neurons) return fail("DelayBuffer::add: post index out of range");
      const uint32_t slot = (uint32_t)((step + std::max<uint32_t>(dl[e], 1)) % kSlots);
      ring[(size_t)slot * n_neurons + post] += w[e];
    }
  }
  return 0;
}

uint64_t or_compact(const int32_t *spikes, uint64_t n, uint32_t *out) {
  uint64_t k = 0;
  for (uint64_t i = 0; i < n; ++i)
    if (spikes[i] != 0) out[k++] = (uint32_t)i;
  return k;
}

int or_kuramoto_rk4(int precision, uint32_t n, const float *theta0, const float *omega, float k,
                    float dt, uint32_t n_steps, float *theta_out, double *r_out) {
  if (n == 0) return fail("empty population");
  if (precision) return kuramoto_rk4<double>(n, theta0, omega, k, dt, n_steps, theta_out, r_out);
  return kuramoto_rk4<float>(n, theta0, omega, k, dt, n_steps, theta_out, r_out);
}

}  // extern "C"
