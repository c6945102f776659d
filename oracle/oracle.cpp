// oracle.cpp -- CPU FP64 restatement of klft's lattice-gauge update-and-measure
// path.  TEST INFRASTRUCTURE ONLY: this file is the checker used by tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg.  Nothing in the
// product (klft_b200/) links or calls it.
//
// Every function cites the reference file:line it restates.  The random
// stream is the project's counter-based Philox4x32-10 (Salmon et al.,
// SC'11), written independently of the GPU code; the stream layout is the
// contract both sides implement (see stream_* below).
//
// Host interchange layout ("AoS site-major", also the C-ABI upload format):
//   U[(((site*Nd + mu)*Nc + i)*Nc + j)] complex<double>,
//   site = x0 + L0*(x1 + L1*(x2 + L2*x3))   (x0 fastest).

#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

using cplx = std::complex<double>;

namespace orc {

// ---------------------------------------------------------------- Philox
static inline void mulhilo(uint32_t a, uint32_t b, uint32_t &hi, uint32_t &lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  hi = (uint32_t)(p >> 32);
  lo = (uint32_t)p;
}

// Philox4x32 with 10 rounds (Random123 constants).
static void philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, c0, hi0, lo0);
    mulhilo(0xCD9E8D57u, c2, hi1, lo1);
    uint32_t n0 = hi1 ^ c1 ^ k0;
    uint32_t n1 = lo1;
    uint32_t n2 = hi0 ^ c3 ^ k1;
    uint32_t n3 = lo0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// Stream kinds (top byte of counter word 3).
enum : uint32_t {
  KIND_METROPOLIS = 1u,  // per (sweep, site): all Nd links x nHits hits in order
  KIND_INIT = 2u,        // per (site, mu): hot-start link
  KIND_MOMENTUM = 3u,    // per (trajectory, site, mu): HMC momentum components
  KIND_HMC_ACCEPT = 4u,  // per trajectory: accept/reject uniform
  KIND_SWAP = 5u,        // per (cycle, pair): replica swap uniform
};

// A sequential stream of uniforms in [0,1):
//   key  = (lo32(seed), hi32(seed) ^ lo32(chain))
//   ctr  = (block, site, step, kind<<24 | sub)
// Each Philox block yields two 53-bit doubles: (w0:w1) then (w2:w3).
struct Stream {
  uint32_t key[2];
  uint32_t ctr[4];
  uint32_t buf[4];
  int avail;  // 0, 1 or 2 doubles left in buf
  Stream(uint64_t seed, uint64_t chain, uint32_t site, uint32_t step, uint32_t kind, uint32_t sub) {
    key[0] = (uint32_t)seed;
    key[1] = (uint32_t)(seed >> 32) ^ (uint32_t)chain;
    ctr[0] = 0; ctr[1] = site; ctr[2] = step; ctr[3] = (kind << 24) | (sub & 0xFFFFFFu);
    avail = 0;
  }
  double next() {
    if (avail == 0) {
      philox(ctr, key, buf);
      ctr[0] += 1;
      avail = 2;
    }
    uint32_t hi, lo;
    if (avail == 2) { hi = buf[0]; lo = buf[1]; } else { hi = buf[2]; lo = buf[3]; }
    avail -= 1;
    uint64_t bits = (((uint64_t)hi << 32) | lo) >> 11;
    return (double)bits * 0x1.0p-53;
  }
  // Kokkos-style drand(start, end) = start + (end - start) * u
  double drand(double a, double b) { return a + (b - a) * next(); }
  // Box-Muller pair from two uniforms
  void gauss2(double &g0, double &g1) {
    double u0 = next();
    double u1 = next();
    double r = std::sqrt(-2.0 * std::log(1.0 - u0));
    double t = 6.283185307179586 * u1;
    g0 = r * std::cos(t);
    g1 = r * std::sin(t);
  }
};

// ---------------------------------------------------------------- SU(N)
template <int NC> struct Mat { cplx a[NC][NC]; };

template <int NC> static inline Mat<NC> zero() {
  Mat<NC> m;
  for (int i = 0; i < NC; ++i) for (int j = 0; j < NC; ++j) m.a[i][j] = cplx(0.0, 0.0);
  return m;
}
template <int NC> static inline Mat<NC> ident() {
  Mat<NC> m = zero<NC>();
  for (int i = 0; i < NC; ++i) m.a[i][i] = cplx(1.0, 0.0);
  return m;
}
// SUN.hpp:28-44  c[i][j] = a[i][0]*b[0][j] + a[i][1]*b[1][j] + ...
template <int NC> static inline Mat<NC> mul(const Mat<NC> &x, const Mat<NC> &y) {
  Mat<NC> c;
  for (int i = 0; i < NC; ++i)
    for (int j = 0; j < NC; ++j) {
      cplx s = x.a[i][0] * y.a[0][j];
      for (int k = 1; k < NC; ++k) s += x.a[i][k] * y.a[k][j];
      c.a[i][j] = s;
    }
  return c;
}
// SUN.hpp:134-146 conj() is the hermitian conjugate
template <int NC> static inline Mat<NC> dag(const Mat<NC> &x) {
  Mat<NC> c;
  for (int i = 0; i < NC; ++i) for (int j = 0; j < NC; ++j) c.a[i][j] = std::conj(x.a[j][i]);
  return c;
}
template <int NC> static inline void addto(Mat<NC> &x, const Mat<NC> &y) {
  for (int i = 0; i < NC; ++i) for (int j = 0; j < NC; ++j) x.a[i][j] += y.a[i][j];
}
template <int NC> static inline Mat<NC> scale(const Mat<NC> &x, double s) {
  Mat<NC> c;
  for (int i = 0; i < NC; ++i) for (int j = 0; j < NC; ++j) c.a[i][j] = x.a[i][j] * s;
  return c;
}
// SUN.hpp:148-157
template <int NC> static inline cplx trace(const Mat<NC> &x) {
  cplx c(0.0, 0.0);
  for (int i = 0; i < NC; ++i) c += x.a[i][i];
  return c;
}

// SUN.hpp:256-340 restoreSUN
static inline Mat<1> restore(const Mat<1> &a) {
  Mat<1> c;
  c.a[0][0] = a.a[0][0] / std::sqrt(a.a[0][0].real() * a.a[0][0].real() + a.a[0][0].imag() * a.a[0][0].imag());
  return c;
}
static inline Mat<2> restore(const Mat<2> &a) {
  Mat<2> c;
  double n = std::sqrt(a.a[0][0].real() * a.a[0][0].real() + a.a[0][0].imag() * a.a[0][0].imag() +
                       a.a[0][1].real() * a.a[0][1].real() + a.a[0][1].imag() * a.a[0][1].imag());
  c.a[0][0] = a.a[0][0] / n; c.a[0][1] = a.a[0][1] / n;
  c.a[1][0] = a.a[1][0] / n; c.a[1][1] = a.a[1][1] / n;
  return c;
}
static inline Mat<3> restore(const Mat<3> &a) {
  Mat<3> c;
  double n0 = std::sqrt((std::conj(a.a[0][0]) * a.a[0][0] + std::conj(a.a[0][1]) * a.a[0][1] +
                         std::conj(a.a[0][2]) * a.a[0][2]).real());
  double n1 = std::sqrt((std::conj(a.a[1][0]) * a.a[1][0] + std::conj(a.a[1][1]) * a.a[1][1] +
                         std::conj(a.a[1][2]) * a.a[1][2]).real());
  for (int j = 0; j < 3; ++j) { c.a[0][j] = a.a[0][j] / n0; c.a[1][j] = a.a[1][j] / n1; }
  c.a[2][0] = std::conj(c.a[0][1] * c.a[1][2] - c.a[0][2] * c.a[1][1]);
  c.a[2][1] = std::conj(c.a[0][2] * c.a[1][0] - c.a[0][0] * c.a[1][2]);
  c.a[2][2] = std::conj(c.a[0][0] * c.a[1][1] - c.a[0][1] * c.a[1][0]);
  c.a[1][0] = std::conj(c.a[2][1] * c.a[0][2] - c.a[2][2] * c.a[0][1]);
  c.a[1][1] = std::conj(c.a[2][2] * c.a[0][0] - c.a[2][0] * c.a[0][2]);
  c.a[1][2] = std::conj(c.a[2][0] * c.a[0][1] - c.a[2][1] * c.a[0][0]);
  return c;
}

// exp(i Q) for a hermitian traceless 3x3 Q by Taylor series with scaling and
// squaring (an independent method from the Cayley-Hamilton form used on the GPU).
static Mat<3> expi_herm3(const Mat<3> &Q) {
  double nrm = 0.0;
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) nrm += std::norm(Q.a[i][j]);
  nrm = std::sqrt(nrm);
  int s = 0;
  while (nrm > 0.25) { nrm *= 0.5; ++s; }
  Mat<3> A;  // A = i Q / 2^s
  double f = std::ldexp(1.0, -s);
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) A.a[i][j] = cplx(0.0, 1.0) * Q.a[i][j] * f;
  Mat<3> R = ident<3>(), T = ident<3>();
  for (int k = 1; k <= 20; ++k) {
    T = scale(mul(T, A), 1.0 / k);
    addto(R, T);
  }
  for (int k = 0; k < s; ++k) R = mul(R, R);
  return R;
}

// Gell-Mann matrices lambda_a (a = 0..7 for lambda_1..lambda_8)
static Mat<3> gellmann(int a) {
  Mat<3> m = zero<3>();
  const cplx I(0.0, 1.0);
  switch (a) {
    case 0: m.a[0][1] = 1.0; m.a[1][0] = 1.0; break;
    case 1: m.a[0][1] = -I; m.a[1][0] = I; break;
    case 2: m.a[0][0] = 1.0; m.a[1][1] = -1.0; break;
    case 3: m.a[0][2] = 1.0; m.a[2][0] = 1.0; break;
    case 4: m.a[0][2] = -I; m.a[2][0] = I; break;
    case 5: m.a[1][2] = 1.0; m.a[2][1] = 1.0; break;
    case 6: m.a[1][2] = -I; m.a[2][1] = I; break;
    case 7: {
      double r = 1.0 / std::sqrt(3.0);
      m.a[0][0] = r; m.a[1][1] = r; m.a[2][2] = -2.0 * r;
    } break;
  }
  return m;
}

// ---------------------------------------------------------------- proposals
enum { PROPOSAL_REFERENCE = 0, PROPOSAL_EXP = 1 };

// SUN.hpp:163-171
static inline void randsun(Mat<1> &r, Stream &g, double delta, int, double) {
  double phi = g.drand(-delta * M_PI, delta * M_PI);
  r.a[0][0] = std::exp(cplx(0.0, phi));
}
// SUN.hpp:174-189
static inline void randsun(Mat<2> &r, Stream &g, double delta, int, double) {
  double alpha = g.drand(0.0, delta * 2 * M_PI);
  double u = g.drand(-1.0, 1.0);
  double theta = g.drand(0.0, 2.0 * M_PI);
  double salpha = std::sin(alpha);
  double n1 = std::sqrt(1.0 - u * u) * std::sin(theta);
  double n2 = std::sqrt(1.0 - u * u) * std::cos(theta);
  r.a[0][0] = cplx(std::cos(alpha), u * salpha);
  r.a[0][1] = cplx(n1 * salpha, n2 * salpha);
  r.a[1][0] = cplx(-r.a[0][1].real(), r.a[0][1].imag());
  r.a[1][1] = cplx(r.a[0][0].real(), -r.a[0][0].imag());
}
// Project SU(3) proposal X = exp(i eps H), H = sum_a h_a lambda_a / 2, h_a ~ N(0,1).
// It has no counterpart in the reference, so its random numbers sit at fixed
// positions of the (sweep, site) stream: hit h of the site (h = mu*nHits + hit)
// takes Philox block h (sub-stream 0); word k gives the Box-Muller pair of
// h_{2k+1}, h_{2k+2} from its two 16-bit halves, u = (k + 1/2) 2^-16 (low half
// for the radius, high half for the angle).  Its accept uniform is word h mod 4
// of block h / 4 of sub-stream 1, (w + 1/2) 2^-32.  A proposal therefore does
// not depend on earlier accept decisions.
struct ExpHit {
  uint32_t key[2], site, step;
  ExpHit(uint64_t seed, uint64_t chain, uint32_t site_, uint32_t step_) : site(site_), step(step_) {
    key[0] = (uint32_t)seed;
    key[1] = (uint32_t)(seed >> 32) ^ (uint32_t)chain;
  }
  void block(uint32_t b, uint32_t out[4], uint32_t sub = 0) const {
    uint32_t ctr[4] = {b, site, step, (KIND_METROPOLIS << 24) | sub};
    philox(ctr, key, out);
  }
  void gauss8(uint32_t h, double g[8]) const {
    uint32_t w[4];
    block(h, w);
    for (int k = 0; k < 4; ++k) {
      const double ua = ((double)(w[k] & 0xFFFFu) + 0.5) * 0x1.0p-16;
      const double ub = ((double)(w[k] >> 16) + 0.5) * 0x1.0p-16;
      const double r = std::sqrt(-2.0 * std::log(ua));
      g[2 * k] = r * std::cos(6.283185307179586 * ub);
      g[2 * k + 1] = r * std::sin(6.283185307179586 * ub);
    }
  }
  double accept_uniform(uint32_t h) const {
    uint32_t w[4];
    block(h >> 2, w, 1);
    return ((double)w[h & 3] + 0.5) * 0x1.0p-32;
  }
};

static Mat<3> exp_proposal(const ExpHit &eh, uint32_t h, double eps) {
  double hh[8];
  eh.gauss8(h, hh);
  Mat<3> H = zero<3>();
  for (int a = 0; a < 8; ++a) {
    Mat<3> l = gellmann(a);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) H.a[i][j] += (0.5 * eps * hh[a]) * l.a[i][j];
  }
  return expi_herm3(H);
}

// SUN.hpp:192-251: reference Gram-Schmidt proposal
static inline void randsun(Mat<3> &r, Stream &g, double delta, int, double) {
  double r1[6], r2[6], norm, fact;
  cplx z1[3], z2[3], z3[3], z;
  while (true) {
    for (int i = 0; i < 6; ++i) r1[i] = g.drand(0, delta);
    norm = std::sqrt(r1[0] * r1[0] + r1[1] * r1[1] + r1[2] * r1[2] + r1[3] * r1[3] + r1[4] * r1[4] + r1[5] * r1[5]);
    if (1.0 != (1.0 + norm)) break;
  }
  fact = 1.0 / norm;
  z1[0] = fact * cplx(r1[0], r1[1]);
  z1[1] = fact * cplx(r1[2], r1[3]);
  z1[2] = fact * cplx(r1[4], r1[5]);
  while (true) {
    while (true) {
      for (int i = 0; i < 6; ++i) r2[i] = g.drand(0, delta);
      norm = std::sqrt(r2[0] * r2[0] + r2[1] * r2[1] + r2[2] * r2[2] + r2[3] * r2[3] + r2[4] * r2[4] + r2[5] * r2[5]);
      if (1.0 != (1.0 + norm)) break;
    }
    fact = 1.0 / norm;
    z2[0] = fact * cplx(r2[0], r2[1]);
    z2[1] = fact * cplx(r2[2], r2[3]);
    z2[2] = fact * cplx(r2[4], r2[5]);
    z = std::conj(z1[0]) * z2[0] + std::conj(z1[1]) * z2[1] + std::conj(z1[2]) * z2[2];
    z2[0] -= z * z1[0];
    z2[1] -= z * z1[1];
    z2[2] -= z * z1[2];
    norm = std::sqrt(z2[0].real() * z2[0].real() + z2[0].imag() * z2[0].imag() + z2[1].real() * z2[1].real() +
                     z2[1].imag() * z2[1].imag() + z2[2].real() * z2[2].real() + z2[2].imag() * z2[2].imag());
    if (1.0 != (1.0 + norm)) break;
  }
  fact = 1.0 / norm;
  z2[0] *= fact; z2[1] *= fact; z2[2] *= fact;
  z3[0] = std::conj((z1[1] * z2[2]) - (z1[2] * z2[1]));
  z3[1] = std::conj((z1[2] * z2[0]) - (z1[0] * z2[2]));
  z3[2] = std::conj((z1[0] * z2[1]) - (z1[1] * z2[0]));
  for (int j = 0; j < 3; ++j) { r.a[0][j] = z1[j]; r.a[1][j] = z2[j]; r.a[2][j] = z3[j]; }
}

// ---------------------------------------------------------------- geometry
// Open boundary (the intent of GaugeField.hpp:168-185 openBC<mu>): links
// U_mu on the slice x_mu = L_mu - 1 are zero and never updated.  -1: periodic.
static int g_open_mu = -1;

struct Geo {
  int nd;
  int L[4];
  long V;
  Geo(int nd_, const int *L_) : nd(nd_) {
    V = 1;
    for (int d = 0; d < 4; ++d) { L[d] = d < nd ? L_[d] : 1; V *= L[d]; }
  }
  long lex(const int x[4]) const {
    long s = 0;
    for (int d = nd - 1; d >= 0; --d) s = s * L[d] + x[d];
    return s;
  }
  bool open_link(long s, int mu) const {
    if (mu != g_open_mu) return false;
    int x[4];
    coords(s, x);
    return x[mu] == L[mu] - 1;
  }
  void coords(long s, int x[4]) const {
    for (int d = 0; d < 4; ++d) x[d] = 0;
    for (int d = 0; d < nd; ++d) { x[d] = (int)(s % L[d]); s /= L[d]; }
  }
  long shift(long s, int d, int k) const {  // s + k e_d (periodic)
    int x[4];
    coords(s, x);
    x[d] = (int)(((long)x[d] + k) % L[d]);
    if (x[d] < 0) x[d] += L[d];
    return lex(x);
  }
};

// PTBC defect (PTBCGaugeField.hpp:30-36, set_defect :187-198): links mu=0 at
// x0 = 0 with x_d in (pos_d + [0, len)) mod L_d for d = 1..Nd-1 carry factor c.
struct Defect {
  int active;
  int len;
  int pos[3];
  double c;
};
static inline double link_factor(const Geo &g, const Defect *df, long s, int mu) {
  if (!df || !df->active || mu != 0) return 1.0;
  int x[4];
  g.coords(s, x);
  if (x[0] != 0) return 1.0;
  for (int d = 1; d < g.nd; ++d) {
    int rel = ((x[d] - df->pos[d - 1]) % g.L[d] + g.L[d]) % g.L[d];
    if (rel >= df->len) return 1.0;
  }
  return df->c;
}

template <int NC> struct Field {
  const Geo &g;
  cplx *U;
  const Defect *df;
  Mat<NC> raw(long s, int mu) const {
    Mat<NC> m;
    const cplx *p = U + ((s * g.nd + mu) * NC) * NC;
    for (int i = 0; i < NC; ++i) for (int j = 0; j < NC; ++j) m.a[i][j] = p[i * NC + j];
    return m;
  }
  // PTBCGaugeField.hpp:209-229 accessor multiplies by the defect factor
  Mat<NC> at(long s, int mu) const {
    Mat<NC> m = raw(s, mu);
    double c = link_factor(g, df, s, mu);
    if (c != 1.0) m = scale(m, c);
    return m;
  }
  void put(long s, int mu, const Mat<NC> &m) const {
    cplx *p = U + ((s * g.nd + mu) * NC) * NC;
    for (int i = 0; i < NC; ++i) for (int j = 0; j < NC; ++j) p[i * NC + j] = m.a[i][j];
  }
};

// GaugeField.hpp:187-237 (3D :389-433, 2D :579-618); PTBC :232-277
template <int NC> static Mat<NC> staple(const Field<NC> &F, long s, int mu) {
  const Geo &g = F.g;
  Mat<NC> temp = zero<NC>();
  long spmu = g.shift(s, mu, 1);
  for (int nu = 0; nu < g.nd; ++nu) {
    if (nu == mu) continue;
    long spnu = g.shift(s, nu, 1);
    addto(temp, mul(mul(F.at(spmu, nu), dag(F.at(spnu, mu))), dag(F.at(s, nu))));
  }
  for (int nu = 0; nu < g.nd; ++nu) {
    if (nu == mu) continue;
    long spmu_mnu = g.shift(spmu, nu, -1);
    long smnu = g.shift(s, nu, -1);
    addto(temp, mul(mul(dag(F.at(spmu_mnu, nu)), dag(F.at(smnu, mu))), F.at(smnu, nu)));
  }
  return temp;
}

// Neumaier's compensated sum: the lattice sums of the checker stay accurate to
// about one rounding of the total at any volume, so that a GPU sum in another
// order is compared with the exact value rather than with a second rounded one.
struct CompSum {
  double s = 0.0, c = 0.0;
  void add(double x) {
    const double t = s + x;
    c += std::fabs(s) >= std::fabs(x) ? (s - t) + x : (x - t) + s;
    s = t;
  }
  double value() const { return s + c; }
};

// GaugePlaquette.hpp:53-85 per site, :125-132 normalisation (returns real part)
template <int NC> static double plaquette(const Field<NC> &F, bool normalize) {
  const Geo &g = F.g;
  CompSum total;
  for (long s = 0; s < g.V; ++s) {
    cplx t(0.0, 0.0);
    for (int mu = 0; mu < g.nd; ++mu)
      for (int nu = 0; nu < g.nd; ++nu) {
        if (nu <= mu) continue;
        Mat<NC> lmu = mul(F.at(s, mu), F.at(g.shift(s, mu, 1), nu));
        Mat<NC> lnu = mul(F.at(s, nu), F.at(g.shift(s, nu, 1), mu));
        for (int a = 0; a < NC; ++a) for (int b = 0; b < NC; ++b) t += lmu.a[a][b] * std::conj(lnu.a[a][b]);
      }
    total.add(t.real());
  }
  double r = total.value();
  if (normalize) r /= (double)g.V * (double)((g.nd * (g.nd - 1) / 2) * NC);
  return r;
}

template <int NC> static Mat<NC> line(const Field<NC> &F, long s, int mu, int len) {
  // WilsonLoop.hpp:61-77 builds lines by right-multiplication from the identity
  Mat<NC> l = ident<NC>();
  long y = s;
  for (int i = 0; i < len; ++i) { l = mul(l, F.at(y, mu)); y = F.g.shift(y, mu, 1); }
  return l;
}

// WilsonLoop.hpp:130-160 (loop per site), :205-244 (normalisation by V*Nc)
template <int NC> static double wilson_mu_nu(const Field<NC> &F, int mu, int nu, int Lmu, int Lnu) {
  const Geo &g = F.g;
  cplx total(0.0, 0.0);
  for (long s = 0; s < g.V; ++s) {
    Mat<NC> wmu = line(F, s, mu, Lmu), wnu = line(F, s, nu, Lnu);
    Mat<NC> lmu = mul(wmu, line(F, g.shift(s, mu, Lmu), nu, Lnu));
    Mat<NC> lnu = mul(wnu, line(F, g.shift(s, nu, Lnu), mu, Lmu));
    cplx t(0.0, 0.0);
    for (int a = 0; a < NC; ++a) for (int b = 0; b < NC; ++b) t += lmu.a[a][b] * std::conj(lnu.a[a][b]);
    total += t;
  }
  for (int d = 0; d < g.nd; ++d) total /= (double)g.L[d];
  total /= (double)NC;
  return total.real();
}

// GaugeVector.hpp:237-262 (get_W_loop_mu_nu, the legacy GaugeVector path), as
// its whole-field steps: set_one + wilson_line (:224-235, right-multiplication
// along the direction), copy, shift_plus (:188-196, out(x) = in(x + dist e_d)),
// UxU / UxUdag (:130-170) and sum_retrace (:213-222); Normalize divides by V*Nc.
template <int NC>
static double wilson_legacy(const Field<NC> &F, int mu, int nu, int Lmu, int Lnu, bool normalize) {
  const Geo &g = F.g;
  std::vector<Mat<NC>> U1(g.V), U2(g.V), U3, U4, tmp(g.V);
  for (long s = 0; s < g.V; ++s) {
    U1[s] = ident<NC>();
    long y = s;
    for (int i = 0; i < Lmu; ++i) { U1[s] = mul(U1[s], F.at(y, mu)); y = g.shift(y, mu, 1); }
    U2[s] = ident<NC>();
    y = s;
    for (int i = 0; i < Lnu; ++i) { U2[s] = mul(U2[s], F.at(y, nu)); y = g.shift(y, nu, 1); }
  }
  U3 = U1;
  U4 = U2;
  for (long s = 0; s < g.V; ++s) tmp[s] = U2[g.shift(s, mu, Lmu)];
  U2 = tmp;
  for (long s = 0; s < g.V; ++s) U1[s] = mul(U1[s], U2[s]);
  for (long s = 0; s < g.V; ++s) tmp[s] = U3[g.shift(s, nu, Lnu)];
  U3 = tmp;
  for (long s = 0; s < g.V; ++s) U1[s] = mul(U1[s], dag(U3[s]));
  for (long s = 0; s < g.V; ++s) U1[s] = mul(U1[s], dag(U4[s]));
  double W = 0.0;
  for (long s = 0; s < g.V; ++s) W += trace(U1[s]).real();
  if (normalize) W /= (double)g.V * (double)NC;
  return W;
}

// One link's hits, Metropolis.hpp:81-107 (reference proposals, U r) or the
// project's exp(i eps H) proposal (X U, accepted products kept unprojected while
// the link's hits run and reunitarised once at the end).
template <int NC>
static uint64_t link_hits(const Field<NC> &F, long s, int mu, double beta, double delta, int nHits, int proposal,
                          double eps, Stream &rng, const ExpHit &eh) {
  const Geo &g = F.g;
  if (g.open_link(s, mu)) return 0;
  const bool expprop = NC == 3 && proposal == PROPOSAL_EXP;
  uint64_t nacc = 0;
  const Mat<NC> S = staple(F, s, mu);
  const double c = link_factor(g, F.df, s, mu);
  Mat<NC> Ucur = F.raw(s, mu);
  bool changed = false;
  for (int hit = 0; hit < nHits; ++hit) {
    const uint32_t h = (uint32_t)(mu * nHits + hit);
    Mat<NC> r;
    if constexpr (NC == 3) {
      if (expprop) r = exp_proposal(eh, h, eps);
      else randsun(r, rng, delta, proposal, eps);
    } else {
      randsun(r, rng, delta, proposal, eps);
    }
    // reference proposals U r (Metropolis.hpp:91); exp(i eps H) proposals X U
    const Mat<NC> Uold = expprop ? Ucur : F.raw(s, mu);
    const Mat<NC> Unew = expprop ? mul(r, Uold) : mul(Uold, r);
    double dS = -(beta / (double)NC) * (trace(mul(Unew, S)).real() - trace(mul(Uold, S)).real());
    if (c != 1.0) dS *= c;
    bool accept = dS < 0.0;
    if (!accept) accept = ((expprop ? eh.accept_uniform(h) : rng.drand(0.0, 1.0)) < std::exp(-dS));
    if (accept) {
      if (expprop) {
        Ucur = Unew;
        changed = true;
      } else {
        F.put(s, mu, restore(Unew));
      }
      ++nacc;
    }
  }
  if (changed) F.put(s, mu, restore(Ucur));
  return nacc;
}

// Metropolis.hpp:73-113 (site functor), :118-178 (sublattice sweep, acceptance
// norm).  The exp(i eps H) proposal has no reference chain: its sweep is 2 Nd
// link passes (mu, p), each updating U_mu(x) at every site of parity
// p = sum_d x_d mod 2 (the links of a pass share no staple link).
template <int NC>
static double metropolis_sweep(const Field<NC> &F, double beta, double delta, int nHits, int proposal, double eps,
                               uint64_t seed, uint64_t chain, uint32_t sweep, uint64_t *nacc_out) {
  const Geo &g = F.g;
  const int nd = g.nd;
  uint64_t nacc = 0;
  if (NC == 3 && proposal == PROPOSAL_EXP) {
    for (int mu = 0; mu < nd; ++mu)
      for (int p = 0; p < 2; ++p) {
#pragma omp parallel for schedule(static) reduction(+ : nacc) if (g.V >= 8192)
        for (long s = 0; s < g.V; ++s) {
          int x[4];
          g.coords(s, x);
          if (((x[0] + x[1] + x[2] + x[3]) & 1) != p) continue;
          Stream rng(seed, chain, (uint32_t)s, sweep, KIND_METROPOLIS, 0);
          const ExpHit eh(seed, chain, (uint32_t)s, sweep);
          nacc += link_hits(F, s, mu, beta, delta, nHits, proposal, eps, rng, eh);
        }
      }
  } else {
    int H[4];
    long Vh = 1;
    for (int d = 0; d < 4; ++d) { H[d] = d < nd ? g.L[d] / 2 : 1; Vh *= H[d]; }
    for (int i = 0; i < (1 << nd); ++i) {
      int bit[4] = {0, 0, 0, 0};
      for (int k = 0; k < nd; ++k) bit[nd - 1 - k] = (i >> k) & 1;  // IndexHelper.hpp:84-93
      // sites of one parity class share no staple link and each reads its own
      // random stream, so the class loop may run on several threads with the
      // same result (the reference runs it as one parallel_for)
#pragma omp parallel for schedule(static) reduction(+ : nacc) if (Vh >= 4096)
      for (long h = 0; h < Vh; ++h) {
        int x[4] = {0, 0, 0, 0};
        long t = h;
        for (int d = 0; d < nd; ++d) { x[d] = 2 * (int)(t % H[d]) + bit[d]; t /= H[d]; }  // IndexHelper.hpp:68-81
        long s = g.lex(x);
        Stream rng(seed, chain, (uint32_t)s, sweep, KIND_METROPOLIS, 0);
        const ExpHit eh(seed, chain, (uint32_t)s, sweep);
        for (int mu = 0; mu < nd; ++mu) nacc += link_hits(F, s, mu, beta, delta, nHits, proposal, eps, rng, eh);
      }
    }
  }
  if (nacc_out) *nacc_out = nacc;
  double norm = 1.0;
  for (int d = 0; d < nd; ++d) norm *= (double)g.L[d];
  norm *= (double)nd;
  norm *= (double)nHits;
  return (double)nacc / norm;
}

// ---------------------------------------------------------------- start
// Haar-random link for the hot start, from the KIND_INIT stream of (site, mu).
static inline void haar(Mat<1> &m, Stream &g) {
  double phi = g.drand(-M_PI, M_PI);
  m.a[0][0] = cplx(std::cos(phi), std::sin(phi));
}
static inline void haar(Mat<2> &m, Stream &g) {
  double q[4];
  g.gauss2(q[0], q[1]);
  g.gauss2(q[2], q[3]);
  double n = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  for (int k = 0; k < 4; ++k) q[k] /= n;
  m.a[0][0] = cplx(q[0], q[3]);
  m.a[0][1] = cplx(q[2], q[1]);
  m.a[1][0] = cplx(-q[2], q[1]);
  m.a[1][1] = cplx(q[0], -q[3]);
}
static inline void haar(Mat<3> &m, Stream &g) {
  // two complex Gaussian rows, Gram-Schmidt, third row = conj(cross)
  cplx r0[3], r1[3];
  for (int j = 0; j < 3; ++j) { double a, b; g.gauss2(a, b); r0[j] = cplx(a, b); }
  for (int j = 0; j < 3; ++j) { double a, b; g.gauss2(a, b); r1[j] = cplx(a, b); }
  double n0 = std::sqrt(std::norm(r0[0]) + std::norm(r0[1]) + std::norm(r0[2]));
  for (int j = 0; j < 3; ++j) r0[j] /= n0;
  cplx z = std::conj(r0[0]) * r1[0] + std::conj(r0[1]) * r1[1] + std::conj(r0[2]) * r1[2];
  for (int j = 0; j < 3; ++j) r1[j] -= z * r0[j];
  double n1 = std::sqrt(std::norm(r1[0]) + std::norm(r1[1]) + std::norm(r1[2]));
  for (int j = 0; j < 3; ++j) r1[j] /= n1;
  for (int j = 0; j < 3; ++j) { m.a[0][j] = r0[j]; m.a[1][j] = r1[j]; }
  m.a[2][0] = std::conj(r0[1] * r1[2] - r0[2] * r1[1]);
  m.a[2][1] = std::conj(r0[2] * r1[0] - r0[0] * r1[2]);
  m.a[2][2] = std::conj(r0[0] * r1[1] - r0[1] * r1[0]);
}

template <int NC> static void init_field(const Field<NC> &F, int hot, uint64_t seed, uint64_t chain) {
  for (long s = 0; s < F.g.V; ++s)
    for (int mu = 0; mu < F.g.nd; ++mu) {
      Mat<NC> m = ident<NC>();
      if (hot) {
        Stream st(seed, chain, (uint32_t)s, 0, KIND_INIT, (uint32_t)mu);
        haar(m, st);
      }
      F.put(s, mu, m);
    }
}

// ---------------------------------------------------------------- HMC
// Algebra components per link: U(1) 1, SU(2) 3, SU(3) 8.
template <int NC> constexpr int ncomp() { return NC == 1 ? 1 : (NC == 2 ? 3 : 8); }

// AdjointGroup.hpp:13-19 (SU(2): (2 Im M01, 2 Re M01, 2 Im M00)), :114-117 (U(1): Im M);
// SU(3): Im Tr(lambda_a M) (the same projection with Gell-Mann generators).
static inline void adj(const Mat<1> &M, double *v) { v[0] = M.a[0][0].imag(); }
static inline void adj(const Mat<2> &M, double *v) {
  v[0] = 2.0 * M.a[0][1].imag();
  v[1] = 2.0 * M.a[0][1].real();
  v[2] = 2.0 * M.a[0][0].imag();
}
static inline void adj(const Mat<3> &M, double *v) {
  for (int a = 0; a < 8; ++a) v[a] = trace(mul(gellmann(a), M)).imag();
}

// AdjointGroup.hpp:98-105 (SU(2): cos|a| + i sin|a| n.sigma), :170-173 (U(1): e^{ia});
// SU(3): exp(i sum_a p_a lambda_a).
static inline Mat<1> expmap(const double *p, double t) {
  Mat<1> m;
  m.a[0][0] = cplx(std::cos(t * p[0]), std::sin(t * p[0]));
  return m;
}
static inline Mat<2> expmap2(const double *p, double t) {
  double a0 = t * p[0], a1 = t * p[1], a2 = t * p[2];
  double alpha = std::sqrt(a0 * a0 + a1 * a1 + a2 * a2);
  Mat<2> m;
  if (alpha == 0.0) return ident<2>();
  double n0 = a0 / alpha, n1 = a1 / alpha, n2 = a2 / alpha;
  double sa = std::sin(alpha), ca = std::cos(alpha);
  m.a[0][0] = cplx(ca, n2 * sa);
  m.a[0][1] = cplx(n1 * sa, n0 * sa);
  m.a[1][0] = cplx(-n1 * sa, n0 * sa);
  m.a[1][1] = cplx(ca, -n2 * sa);
  return m;
}
static inline Mat<3> expmap3(const double *p, double t) {
  Mat<3> Q = zero<3>();
  for (int a = 0; a < 8; ++a) {
    Mat<3> l = gellmann(a);
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q.a[i][j] += (t * p[a]) * l.a[i][j];
  }
  return expi_herm3(Q);
}
template <int NC> static inline Mat<NC> expmapN(const double *p, double t);
template <> inline Mat<1> expmapN<1>(const double *p, double t) { return expmap(p, t); }
template <> inline Mat<2> expmapN<2>(const double *p, double t) { return expmap2(p, t); }
template <> inline Mat<3> expmapN<3>(const double *p, double t) { return expmap3(p, t); }

// Generator normalisation of the HMC maps: 1 = the reference's (Pauli /
// Gell-Mann), 1/2 = t_a / 2.  With t_a / 2 the force is (beta/Nc) Im Tr(t_a U S) / 2
// and the update exp(i dt sum_a p_a t_a / 2).
static double g_gen_scale = 1.0;

// GaugeMonomial.hpp:27-37: F(x,mu) = (beta/Nc) Adj(U_mu(x) S_mu(x))
template <int NC> static void gauge_force(const Field<NC> &F, double beta, double *frc) {
  const int nc = ncomp<NC>();
  const double fs = (beta / (double)NC) * g_gen_scale;
#pragma omp parallel for schedule(static) if (F.g.V >= 4096)
  for (long s = 0; s < F.g.V; ++s)
    for (int mu = 0; mu < F.g.nd; ++mu) {
      Mat<NC> M = mul(F.at(s, mu), staple(F, s, mu));
      double v[8];
      adj(M, v);
      for (int a = 0; a < nc; ++a) frc[(s * F.g.nd + mu) * nc + a] = fs * v[a];
    }
}

// GaugeMonomial.hpp:19-25: H_gauge = -(beta/Nc) * sum_x sum_{mu<nu} Re Tr P_{mu nu}
template <int NC> static double gauge_action(const Field<NC> &F, double beta) {
  return -(beta / (double)NC) * plaquette(F, false);
}

// HamiltonianField.hpp:40-48
static double kinetic(const double *P, long n) {
  CompSum k;
  for (long i = 0; i < n; ++i) k.add(0.5 * P[i] * P[i]);
  return k.value();
}

template <int NC> static void momenta(const Geo &g, double *P, uint64_t seed, uint64_t chain, uint32_t traj) {
  const int nc = ncomp<NC>();
#pragma omp parallel for schedule(static) if (g.V >= 4096)
  for (long s = 0; s < g.V; ++s)
    for (int mu = 0; mu < g.nd; ++mu) {
      Stream st(seed, chain, (uint32_t)s, traj, KIND_MOMENTUM, (uint32_t)mu);
      double gs[8];
      for (int k = 0; k < (nc + 1) / 2; ++k) st.gauss2(gs[2 * k], gs[2 * k + 1]);
      for (int a = 0; a < nc; ++a) P[(s * g.nd + mu) * nc + a] = gs[a];
    }
}

// HamiltonianField.hpp:23-38
template <int NC> static void update_momentum(const Field<NC> &F, double *P, double *frc, double beta, double dt) {
  const int nc = ncomp<NC>();
  gauge_force(F, beta, frc);
  for (long i = 0; i < F.g.V * F.g.nd * nc; ++i) P[i] -= dt * frc[i];
}
template <int NC> static void update_gauge(const Field<NC> &F, const double *P, double dt) {
  const int nc = ncomp<NC>();
#pragma omp parallel for schedule(static) if (F.g.V >= 4096)
  for (long s = 0; s < F.g.V; ++s)
    for (int mu = 0; mu < F.g.nd; ++mu)
      F.put(s, mu, mul(expmapN<NC>(P + (s * F.g.nd + mu) * nc, dt * g_gen_scale), F.raw(s, mu)));
}

enum { INTEGRATOR_REFERENCE_LEAPFROG = 0, INTEGRATOR_LEAPFROG = 1, INTEGRATOR_OMELYAN = 2 };

// Integrator.hpp:26-53 (reference leapfrog: n_steps+1 gauge updates of dtau = tau/n_steps),
// the standard n-step leapfrog, and the 2nd-order minimum-norm (Omelyan) scheme.
template <int NC>
static void integrate(const Field<NC> &F, double *P, double beta, double tau, int nsteps, int integrator) {
  const int nc = ncomp<NC>();
  std::vector<double> frc((size_t)F.g.V * F.g.nd * nc);
  const double dt = tau / (double)nsteps;
  if (integrator == INTEGRATOR_REFERENCE_LEAPFROG) {
    update_momentum(F, P, frc.data(), beta, dt / 2.0);
    update_gauge(F, P, dt);
    for (int i = 0; i < nsteps; ++i) {
      update_momentum(F, P, frc.data(), beta, dt);
      update_gauge(F, P, dt);
    }
    update_momentum(F, P, frc.data(), beta, dt / 2.0);
  } else if (integrator == INTEGRATOR_LEAPFROG) {
    update_momentum(F, P, frc.data(), beta, dt / 2.0);
    for (int i = 0; i < nsteps; ++i) {
      update_gauge(F, P, dt);
      update_momentum(F, P, frc.data(), beta, i == nsteps - 1 ? dt / 2.0 : dt);
    }
  } else {
    const double lam = 0.1931833275037836;
    for (int i = 0; i < nsteps; ++i) {
      update_momentum(F, P, frc.data(), beta, lam * dt);
      update_gauge(F, P, dt / 2.0);
      update_momentum(F, P, frc.data(), beta, (1.0 - 2.0 * lam) * dt);
      update_gauge(F, P, dt / 2.0);
      update_momentum(F, P, frc.data(), beta, lam * dt);
    }
  }
#pragma omp parallel for schedule(static) if (F.g.V >= 4096)
  for (long s = 0; s < F.g.V; ++s)
    for (int mu = 0; mu < F.g.nd; ++mu)
      if (!F.g.open_link(s, mu)) F.put(s, mu, restore(F.raw(s, mu)));
}

// HMC.hpp:48-71: refresh P, H_old, integrate, H_new, accept/reject
template <int NC>
static int hmc_trajectory(const Field<NC> &F, double beta, double tau, int nsteps, int integrator, uint64_t seed,
                          uint64_t chain, uint32_t traj, double *dH_out, double *P_out) {
  const int nc = ncomp<NC>();
  const size_t n = (size_t)F.g.V * F.g.nd * nc;
  std::vector<double> P(n);
  momenta<NC>(F.g, P.data(), seed, chain, traj);
  std::vector<cplx> save(F.U, F.U + (size_t)F.g.V * F.g.nd * NC * NC);
  const double k_old = kinetic(P.data(), (long)n);
  const double g_old = gauge_action(F, beta);
  integrate(F, P.data(), beta, tau, nsteps, integrator);
  const double k_new = kinetic(P.data(), (long)n);
  const double g_new = gauge_action(F, beta);
  double dH = 0.0;
  dH += k_new - k_old;
  dH += g_new - g_old;
  int accept = 1;
  if (dH > 0.0) {
    Stream st(seed, chain, 0u, traj, KIND_HMC_ACCEPT, 0);
    if (st.next() > std::exp(-dH)) accept = 0;
  }
  if (!accept) std::copy(save.begin(), save.end(), F.U);
  if (dH_out) *dH_out = dH;
  if (P_out) std::copy(P.begin(), P.end(), P_out);
  return accept;
}

// ---------------------------------------------------------------- PTBC swap
// Per-lattice sums over defect plaquettes grouped by how many defect links they
// hold: out[k-1] = sum_{P: n(P)=k} s_P(U), s_P = -(beta/Nc) Re Tr U_P (raw links).
template <int NC> static void defect_sums(const Field<NC> &F, const Defect &df, double beta, double out[2]) {
  Defect probe = df;
  probe.c = 0.5;  // any c != 1 marks defect links
  out[0] = out[1] = 0.0;
  const Geo &g = F.g;
  Field<NC> R{F.g, F.U, nullptr};
  for (long s = 0; s < g.V; ++s)
    for (int mu = 0; mu < g.nd; ++mu)
      for (int nu = mu + 1; nu < g.nd; ++nu) {
        long spmu = g.shift(s, mu, 1), spnu = g.shift(s, nu, 1);
        int k = (link_factor(g, &probe, s, mu) != 1.0) + (link_factor(g, &probe, spmu, nu) != 1.0) +
                (link_factor(g, &probe, spnu, mu) != 1.0) + (link_factor(g, &probe, s, nu) != 1.0);
        if (k == 0) continue;
        Mat<NC> lmu = mul(R.raw(s, mu), R.raw(spmu, nu));
        Mat<NC> lnu = mul(R.raw(s, nu), R.raw(spnu, mu));
        cplx t(0.0, 0.0);
        for (int a = 0; a < NC; ++a) for (int b = 0; b < NC; ++b) t += lmu.a[a][b] * std::conj(lnu.a[a][b]);
        out[k - 1] += -(beta / (double)NC) * t.real();
      }
}

}  // namespace orc

// ================================================================ C entry points
using namespace orc;

#define DISPATCH_NC(nc, CALL) \
  switch (nc) {               \
    case 1: { constexpr int NC = 1; CALL; } break; \
    case 2: { constexpr int NC = 2; CALL; } break; \
    case 3: { constexpr int NC = 3; CALL; } break; \
    default: return -1;       \
  }

static Defect make_defect(const int *dparams_i, double c) {
  Defect d{0, 1, {0, 0, 0}, 1.0};
  if (dparams_i) {
    d.active = 1;
    d.len = dparams_i[0];
    d.pos[0] = dparams_i[1]; d.pos[1] = dparams_i[2]; d.pos[2] = dparams_i[3];
    d.c = c;
  }
  return d;
}

extern "C" {

int oracle_philox(const uint32_t *ctr, const uint32_t *key, uint32_t *out) {
  philox(ctr, key, out);
  return 0;
}

int oracle_uniforms(uint64_t seed, uint64_t chain, uint32_t site, uint32_t step, uint32_t kind, uint32_t sub, int n,
                    double *out) {
  Stream st(seed, chain, site, step, kind, sub);
  for (int i = 0; i < n; ++i) out[i] = st.next();
  return 0;
}

void oracle_set_open_boundary(int mu) { g_open_mu = mu; }

// HMC generators for the following calls: 0 = the reference's, 1 = t_a / 2
void oracle_set_generators(int half) { g_gen_scale = half ? 0.5 : 1.0; }

// The Lie-algebra maps on one matrix (interleaved re/im, row major): Adj(M)
// and exp(t p) (the reference normalisation), for pinning against klft's code.
int oracle_adjoint(int nc, const double *M, double *v) {
  DISPATCH_NC(nc, ({
    Mat<NC> m;
    for (int i = 0; i < NC; ++i) for (int j = 0; j < NC; ++j) m.a[i][j] = cplx(M[2 * (i * NC + j)], M[2 * (i * NC + j) + 1]);
    adj(m, v);
  }));
  return 0;
}
int oracle_expmap(int nc, const double *p, double t, double *M) {
  DISPATCH_NC(nc, ({
    const Mat<NC> m = expmapN<NC>(p, t);
    for (int i = 0; i < NC; ++i)
      for (int j = 0; j < NC; ++j) { M[2 * (i * NC + j)] = m.a[i][j].real(); M[2 * (i * NC + j) + 1] = m.a[i][j].imag(); }
  }));
  return 0;
}

int oracle_init(int nc, int nd, const int *L, int hot, uint64_t seed, uint64_t chain, double *U) {
  Geo g(nd, L);
  DISPATCH_NC(nc, (init_field<NC>(Field<NC>{g, (cplx *)U, nullptr}, hot, seed, chain)));
  return 0;
}

int oracle_staple_field(int nc, int nd, const int *L, const double *U, double *out) {
  Geo g(nd, L);
  DISPATCH_NC(nc, ({
    Field<NC> F{g, (cplx *)U, nullptr};
    Field<NC> O{g, (cplx *)out, nullptr};
    for (long s = 0; s < g.V; ++s)
      for (int mu = 0; mu < nd; ++mu) O.put(s, mu, staple(F, s, mu));
  }));
  return 0;
}

int oracle_plaquette(int nc, int nd, const int *L, const double *U, int normalize, double *out) {
  Geo g(nd, L);
  DISPATCH_NC(nc, (*out = plaquette(Field<NC>{g, (cplx *)U, nullptr}, normalize != 0)));
  return 0;
}

// pairs: n pairs (Lmu, Lnu); out: n values
int oracle_wilson_mu_nu(int nc, int nd, const int *L, const double *U, int mu, int nu, const int *pairs, int n,
                        double *out) {
  Geo g(nd, L);
  DISPATCH_NC(nc, ({
    Field<NC> F{g, (cplx *)U, nullptr};
    for (int k = 0; k < n; ++k) out[k] = wilson_mu_nu(F, mu, nu, pairs[2 * k], pairs[2 * k + 1]);
  }));
  return 0;
}

int oracle_wilson_legacy(int nc, int nd, const int *L, const double *U, int mu, int nu, int Lmu, int Lnu,
                         int normalize, double *out) {
  Geo g(nd, L);
  DISPATCH_NC(nc, (*out = wilson_legacy(Field<NC>{g, (cplx *)U, nullptr}, mu, nu, Lmu, Lnu, normalize != 0)));
  return 0;
}

// WilsonLoop.hpp:250-304: average over mu = 0..Nd-2 of W(mu, Nd-1)
int oracle_wilson_temporal(int nc, int nd, const int *L, const double *U, const int *pairs, int n, double *out) {
  Geo g(nd, L);
  DISPATCH_NC(nc, ({
    Field<NC> F{g, (cplx *)U, nullptr};
    for (int k = 0; k < n; ++k) {
      double w = 0.0;
      for (int mu = 0; mu < nd - 1; ++mu) w += wilson_mu_nu(F, mu, nd - 1, pairs[2 * k], pairs[2 * k + 1]);
      out[k] = w / (double)(nd - 1);
    }
  }));
  return 0;
}

// dparams: NULL or {len, pos1, pos2, pos3}; defect_c is the factor on defect links
int oracle_metropolis(int nc, int nd, const int *L, double *U, double beta, double delta, int nHits, int proposal,
                      double eps, uint64_t seed, uint64_t chain, uint32_t sweep0, int nsweeps, const int *dparams,
                      double defect_c, double *acc_out) {
  Geo g(nd, L);
  Defect df = make_defect(dparams, defect_c);
  DISPATCH_NC(nc, ({
    Field<NC> F{g, (cplx *)U, &df};
    for (int k = 0; k < nsweeps; ++k)
      acc_out[k] = metropolis_sweep(F, beta, delta, nHits, proposal, eps, seed, chain, sweep0 + (uint32_t)k, nullptr);
  }));
  return 0;
}

int oracle_expi_su3(const double *Q, double *out) {
  Mat<3> q;
  for (int i = 0; i < 9; ++i) q.a[i / 3][i % 3] = cplx(Q[2 * i], Q[2 * i + 1]);
  Mat<3> r = expi_herm3(q);
  for (int i = 0; i < 9; ++i) { out[2 * i] = r.a[i / 3][i % 3].real(); out[2 * i + 1] = r.a[i / 3][i % 3].imag(); }
  return 0;
}

int oracle_gauge_force(int nc, int nd, const int *L, const double *U, double beta, double *frc) {
  Geo g(nd, L);
  DISPATCH_NC(nc, (gauge_force(Field<NC>{g, (cplx *)U, nullptr}, beta, frc)));
  return 0;
}

int oracle_momenta(int nc, int nd, const int *L, uint64_t seed, uint64_t chain, uint32_t traj, double *P) {
  Geo g(nd, L);
  DISPATCH_NC(nc, (momenta<NC>(g, P, seed, chain, traj)));
  return 0;
}

int oracle_gauge_action(int nc, int nd, const int *L, const double *U, double beta, double *out) {
  Geo g(nd, L);
  DISPATCH_NC(nc, (*out = gauge_action(Field<NC>{g, (cplx *)U, nullptr}, beta)));
  return 0;
}

// Integrate one trajectory from given momenta (P updated in place), without accept/reject.
int oracle_integrate(int nc, int nd, const int *L, double *U, double *P, double beta, double tau, int nsteps,
                     int integrator) {
  Geo g(nd, L);
  DISPATCH_NC(nc, (integrate(Field<NC>{g, (cplx *)U, nullptr}, P, beta, tau, nsteps, integrator)));
  return 0;
}

int oracle_hmc(int nc, int nd, const int *L, double *U, double beta, double tau, int nsteps, int integrator,
               uint64_t seed, uint64_t chain, uint32_t traj0, int ntraj, double *dH, int *acc) {
  Geo g(nd, L);
  DISPATCH_NC(nc, ({
    Field<NC> F{g, (cplx *)U, nullptr};
    for (int k = 0; k < ntraj; ++k)
      acc[k] = hmc_trajectory(F, beta, tau, nsteps, integrator, seed, chain, traj0 + (uint32_t)k, &dH[k], nullptr);
  }));
  return 0;
}

int oracle_defect_sums(int nc, int nd, const int *L, const double *U, const int *dparams, double beta, double *out) {
  Geo g(nd, L);
  Defect df = make_defect(dparams, 0.5);
  DISPATCH_NC(nc, (defect_sums(Field<NC>{g, (cplx *)U, nullptr}, df, beta, out)));
  return 0;
}

// Action S_c(U) = -(beta/Nc) sum_P w_c(P) Re Tr U_P with link factors (defect-weighted plaquettes)
int oracle_defect_action(int nc, int nd, const int *L, const double *U, const int *dparams, double c, double beta,
                         double *out) {
  Geo g(nd, L);
  Defect df = make_defect(dparams, c);
  DISPATCH_NC(nc, (*out = -(beta / (double)NC) * plaquette(Field<NC>{g, (cplx *)U, &df}, false)));
  return 0;
}

// Replica swap (project definition; the reference has a defect field but no swap).
// Replica lattice r holds label label_of_rep[r] (coefficient c[label]).  For k =
// 0..nrep-2 the lattices a, b holding labels k, k+1 swap labels with probability
// min(1, exp(-dS)), dS = sum_{n=1,2} (c_k^n - c_{k+1}^n) (A_n(b) - A_n(a)), where
// A[2r + n - 1] = sum over plaquettes of lattice r with n defect links of
// s_P = -(beta/Nc) Re Tr U_P.  The uniform of pair k comes from the (cycle,
// site = k) KIND_SWAP stream of chain 0.
int oracle_ptbc_swap(int nrep, const double *c, const double *A, int *label_of_rep, uint64_t seed, uint32_t cycle,
                     int *accepted) {
  std::vector<int> rep_of_label(nrep);
  for (int r = 0; r < nrep; ++r) rep_of_label[label_of_rep[r]] = r;
  for (int k = 0; k + 1 < nrep; ++k) {
    const int a = rep_of_label[k], b = rep_of_label[k + 1];
    double dS = 0.0;
    dS += (c[k] - c[k + 1]) * (A[2 * b] - A[2 * a]);
    dS += (c[k] * c[k] - c[k + 1] * c[k + 1]) * (A[2 * b + 1] - A[2 * a + 1]);
    bool acc = dS < 0.0;
    if (!acc) {
      Stream st(seed, 0, (uint32_t)k, cycle, KIND_SWAP, 0);
      acc = st.next() < std::exp(-dS);
    }
    accepted[k] = acc ? 1 : 0;
    if (acc) {
      rep_of_label[k] = b;
      rep_of_label[k + 1] = a;
      label_of_rep[a] = k + 1;
      label_of_rep[b] = k;
    }
  }
  return 0;
}

int oracle_unitarity(int nc, int nd, const int *L, const double *U, double *out) {
  Geo g(nd, L);
  double worst = 0.0;
  DISPATCH_NC(nc, ({
    Field<NC> F{g, (cplx *)U, nullptr};
    for (long s = 0; s < g.V; ++s)
      for (int mu = 0; mu < nd; ++mu) {
        Mat<NC> m = mul(dag(F.raw(s, mu)), F.raw(s, mu));
        double e = 0.0;
        for (int i = 0; i < NC; ++i)
          for (int j = 0; j < NC; ++j) e += std::norm(m.a[i][j] - (i == j ? cplx(1.0, 0.0) : cplx(0.0, 0.0)));
        worst = std::max(worst, std::sqrt(e));
      }
  }));
  *out = worst;
  return 0;
}

}  // extern "C"
