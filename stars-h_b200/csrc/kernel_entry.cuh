// Device evaluation of one kernel-matrix entry, shared by the tile
// generator, the fused generation-and-sketch kernel and the error kernel.
//
// Each family computes the same expression, in the same operation order,
// as the reference kernel of that name (src/applications/spatial/
// kernel_{exp,sqrexp,matern,matern2}.c, electrostatics/
// kernel_coulomb_potential.c, electrodynamics/kernel_{sin,cos}.c,
// mesh_deformation/virus.c + kernels_rbf.c), so that generated blocks agree
// with the reference to a few ulp: the squared distance is accumulated
// dimension by dimension without FMA contraction, and divisions are true
// IEEE divisions.  The Matérn families need K_nu, which the reference takes
// from GSL; bessel_knu() below is this library's own implementation.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace b200 {

// Families (values of STARSH_B200_FAMILY_* in starsh-b200.h).
enum : int {
    FAM_EXP = 1, FAM_SQREXP = 2, FAM_MATERN = 3, FAM_MATERN2 = 4,
    FAM_COULOMB = 5, FAM_SIN = 6, FAM_COS = 7, FAM_RBF = 8
};

// Everything a device generator needs: family parameters and device
// pointers to the coordinates and the cluster pivots.
struct DevKernel {
    int family;
    int ndim;
    int aos;          // RBF: point-major coordinates
    int rbf_kind;
    int isreg;
    int zero_mode;    // Coulomb: r = 0 gives `diag` instead of 0
    double sigma, beta, nu, noise;
    double matern_coef, matern_scale;
    int matern_half;          // 1, 2, 3 for nu = 1/2, 3/2, 5/2; else 0
    // Matérn with other nu: polynomial pieces of x^nu e^x K_nu(x) on the
    // eighths of [2^E, 2^(E+1)), kMaternTabEmin <= E < kMaternTabEmin +
    // kMaternTabIntervals (device, 16-byte aligned, or null)
    const double *matern_tab;
    double inv_neg_beta;      // -1/beta (exp)
    double inv_neg_2beta2;    // 1/((-2 beta) beta) (square exponential)
    double wave_k, diag;
    double rad, reg;
    const double *row_pt;     // coordinates of the row point set
    const double *col_pt;     // coordinates of the column point set
    long long row_count, col_count;
    const long long *row_piv; // cluster pivots (STARSH_int)
    const long long *col_piv;
};

// Matérn table: kMaternTabIntervals dyadic intervals covering
// [2^-10, 1024), each cut into kMaternTabSub equal pieces (the top three
// mantissa bits of x), each piece a polynomial of degree kMaternTabDeg in
// the piece's own variable u in [-1, 1), monomial coefficients, stored
// kMaternTabStride doubles apart (the last slot zero).  The function is
// analytic except at x = 0, which lies at u <= -17 for every piece: a
// Bernstein ellipse of rho >= 17 + 12 sqrt 2 ~ 34 at every scale, so
// degree 10 interpolates it to rounding (<= 2.1e-16 relative against
// mpmath for 0.2 <= nu <= 4.7, Horner in double).
constexpr int kMaternTabDeg = 10;
constexpr int kMaternTabSub = 8;
constexpr int kMaternTabStride = 12;
constexpr int kMaternTabEmin = -10;
constexpr int kMaternTabIntervals = 20;
constexpr int kMaternTabPieces = kMaternTabIntervals * kMaternTabSub;
constexpr double kMaternTabLo = 0.0009765625;   // 2^kMaternTabEmin

// Taylor coefficients of 1/Gamma(1+z) about z = 0 (a_0 = 1, a_1 = Euler's
// gamma, ...), computed with mpmath at 50 digits by
// stars-h_b200/csrc/gen_rgamma_coeffs.py.
__device__ __constant__ static const double kRGammaCoef[29] = {
    1.0,
    0.5772156649015328606065121,
    -0.6558780715202538810770195,
    -0.04200263503409523552900393,
    0.1665386113822914895017008,
    -0.0421977345555443367482083,
    -0.009621971527876973562114922,
    0.00721894324666309954239501,
    -0.001165167591859065112113971,
    -0.00021524167411495097281573,
    0.0001280502823881161861531986,
    -0.00002013485478078823865568939,
    -0.000001250493482142670657345359,
    0.00000113302723198169588237413,
    -0.0000002056338416977607103450154,
    6.116095104481415817862499e-9,
    5.002007644469222930055665e-9,
    -1.181274570487020144588127e-9,
    1.04342671169110051049154e-10,
    7.782263439905071254049937e-12,
    -3.696805618642205708187816e-12,
    5.100370287454475979015481e-13,
    -2.05832605356650678322243e-14,
    -5.348122539423017982370017e-15,
    1.226778628238260790158894e-15,
    -1.181259301697458769513765e-16,
    1.186692254751600332579777e-18,
    1.412380655318031781555804e-18,
    -2.298745684435370206592479e-19,
};

// K_mu(x) and K_{mu+1}(x) for |mu| <= 1/2, 0 < x <= 2, by Temme's series
// (N. M. Temme, J. Comput. Phys. 19 (1975) 324-337):
//   K_mu     = sum_k c_k f_k,      K_{mu+1} = (2/x) sum_k c_k h_k,
//   c_k = (x^2/4)^k / k!,
//   f_0 = (mu pi / sin(mu pi)) [cosh(s) G1 + sinh(s)/s * ln(2/x) G2],
//         s = mu ln(2/x),
//   p_0 = (x/2)^-mu Gamma(1+mu) / 2,  q_0 = (x/2)^mu Gamma(1-mu) / 2,
//   f_k = (k f_{k-1} + p_{k-1} + q_{k-1}) / (k^2 - mu^2),
//   p_k = p_{k-1} / (k - mu),  q_k = q_{k-1} / (k + mu),  h_k = p_k - k f_k,
// with G1 = (1/Gamma(1-mu) - 1/Gamma(1+mu)) / (2 mu) and
// G2 = (1/Gamma(1-mu) + 1/Gamma(1+mu)) / 2 taken from the odd and even
// parts of the power series of 1/Gamma(1+z), which avoids the cancellation
// of the difference quotient at small mu.
__device__ inline void bessel_k_temme(double mu, double x, double *kmu,
                                      double *kmu1)
{
    double g1 = 0.0, g2 = 0.0, mu2 = mu * mu, pw = 1.0;
    // even coefficients -> G2, odd coefficients -> -G1
    #pragma unroll
    for (int j = 0; j < 29; j += 2) {
        g2 += kRGammaCoef[j] * pw;
        if (j + 1 < 29) g1 -= kRGammaCoef[j + 1] * pw;
        pw *= mu2;
    }
    // 1/Gamma(1+mu) = G2 - mu*G1 ; 1/Gamma(1-mu) = G2 + mu*G1
    const double rg_plus = g2 - mu * g1;
    const double rg_minus = g2 + mu * g1;
    const double half_x = 0.5 * x;
    const double lg = -log(half_x);               // ln(2/x)
    const double s = mu * lg;
    const double pimu = M_PI * mu;
    const double fact = fabs(pimu) < 1e-15 ? 1.0 : pimu / sin(pimu);
    const double shs = fabs(s) < 1e-15 ? 1.0 : sinh(s) / s;
    double f = fact * (g1 * cosh(s) + g2 * lg * shs);
    const double e = exp(s);                      // (x/2)^-mu
    double p = 0.5 * e / rg_plus;
    double q = 0.5 / (e * rg_minus);
    double c = 1.0;
    const double c_step = half_x * half_x;
    double sum = f, sum1 = p;
    for (int k = 1; k < 500; ++k) {
        const double dk = (double)k;
        f = (dk * f + p + q) / (dk * dk - mu2);
        c *= c_step / dk;
        p /= (dk - mu);
        q /= (dk + mu);
        const double t = c * f;
        sum += t;
        sum1 += c * (p - dk * f);
        if (fabs(t) < 1e-17 * fabs(sum)) break;
    }
    *kmu = sum;
    *kmu1 = sum1 * (2.0 / x);
}

// K_nu(x) for x > 2 from the integral K_nu(x) = int_0^inf exp(-x cosh t)
// cosh(nu t) dt.  With s = sqrt(2x) sinh(t/2):
//   e^x K_nu(x) = int_0^inf e^{-s^2} cosh(2 nu asinh(y)) 2 / sqrt(2x+s^2) ds,
//   y = s / sqrt(2x),
// an integrand analytic in the strip |Im s| < d = sqrt(2x) with Gaussian
// decay, for which the trapezoidal rule converges geometrically
// (L. N. Trefethen and J. A. C. Weideman, SIAM Review 56 (2014) 385-458).
// On a line Im s = c the Gaussian grows like e^{c^2}, so the error is about
// exp(-2 pi c / h + c^2) for c <= d; h = min(0.49, 2 pi d / (41 + d^2))
// keeps it below ~1e-17 (checked against mpmath to 1e-14 relative for
// 0.1 <= nu <= 4.7, 2 < x <= 300).  Nodes stop where e^{-s^2} < 1e-19.
// e^x K_nu(x) for x > 2 (the integral below without its factor e^-x),
// with the step divided by `refine` (1 in the generators; the table
// builder takes 2, for node values limited by rounding only).
__device__ inline double bessel_k_large_scaled(double nu, double x,
                                               double refine)
{
    const double two_x = 2.0 * x;
    const double d = sqrt(two_x);
    const double h = fmin(0.49, 2.0 * M_PI * d / (41.0 + two_x)) / refine;
    const double inv_d = 1.0 / d;
    double sum = 0.0;
    for (int k = 0; k < 256; ++k) {
        const double s = k * h;
        const double w = exp(-s * s);
        if (w < 1e-19) break;
        const double y = s * inv_d;
        const double a = y + sqrt(1.0 + y * y);   // exp(asinh(y))
        const double ap = exp(2.0 * nu * log(a));  // a^(2 nu)
        const double g = 0.5 * (ap + 1.0 / ap) * 2.0 / sqrt(two_x + s * s);
        sum += (k == 0 ? 0.5 : 1.0) * w * g;
    }
    return h * sum;
}

__device__ inline double bessel_k_large(double nu, double x)
{
    return bessel_k_large_scaled(nu, x, 1.0) * exp(-x);
}

// x^nu e^x K_nu(x) for 2^-10 <= x < 1024 from the problem's table.  With
// x = 2^E (1 + (j + f) / 8), j the top three mantissa bits and f in [0, 1)
// the other 49, the piece is 8 (E - kMaternTabEmin) + j (the high word
// shifted right by 17 holds the biased exponent and j) and u = 2 f - 1,
// formed exactly from the mantissa bits; Horner's rule sums the piece.
__device__ __forceinline__ double matern_tab_eval(const double *tab, double x)
{
    const int hi = __double2hiint(x), lo = __double2loint(x);
    const int piece = (hi >> 17) - ((1023 + kMaternTabEmin) << 3);
    // 1 + f: the low 49 mantissa bits moved to the top, exponent of 1.0
    const double z = __hiloint2double(
        0x3FF00000 | (int)(__funnelshift_l((unsigned)lo, (unsigned)hi, 3) & 0x000FFFFFu),
        (int)((unsigned)lo << 3));
    const double u = fma(z, 2.0, -3.0);
    const double2 *c = reinterpret_cast<const double2 *>(
        tab + (size_t)piece * kMaternTabStride);
    const double2 c01 = __ldg(c), c23 = __ldg(c + 1), c45 = __ldg(c + 2),
                  c67 = __ldg(c + 3), c89 = __ldg(c + 4), c10 = __ldg(c + 5);
    static_assert(kMaternTabDeg == 10 && kMaternTabStride == 12,
                  "Horner chain written for degree 10");
    double p = c10.x;
    p = fma(p, u, c89.y);
    p = fma(p, u, c89.x);
    p = fma(p, u, c67.y);
    p = fma(p, u, c67.x);
    p = fma(p, u, c45.y);
    p = fma(p, u, c45.x);
    p = fma(p, u, c23.y);
    p = fma(p, u, c23.x);
    p = fma(p, u, c01.y);
    return fma(p, u, c01.x);
}

// K_nu(x), nu >= 0, x > 0.  Small arguments: Temme's series at
// mu = nu - round(nu) and upward recurrence
// K_{m+1} = K_{m-1} + (2 m / x) K_m; large arguments: the integral above.
__device__ inline double bessel_knu(double nu, double x)
{
    if (x > 2.0) return bessel_k_large(nu, x);
    const int nl = (int)(nu + 0.5);
    const double mu = nu - nl;
    double k0, k1;
    bessel_k_temme(mu, x, &k0, &k1);
    for (int i = 1; i <= nl; ++i) {
        const double k2 = k0 + (2.0 * (mu + i) / x) * k1;
        k0 = k1;
        k1 = k2;
    }
    return k0;
}

// Squared distance accumulated as the reference does: tmp = a - b;
// dist += tmp*tmp, one dimension after another, no fused multiply-add.
__device__ __forceinline__ double sq_dist(const DevKernel &K, long long ir,
                                          long long jc)
{
    double dist = 0.0;
    if (K.aos) {
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double t = __dsub_rn(K.row_pt[3 * ir + d],
                                       K.col_pt[3 * jc + d]);
            dist = __dadd_rn(dist, __dmul_rn(t, t));
        }
    } else {
        for (int d = 0; d < K.ndim; ++d) {
            const double t = __dsub_rn(K.row_pt[d * K.row_count + ir],
                                       K.col_pt[d * K.col_count + jc]);
            dist = __dadd_rn(dist, __dmul_rn(t, t));
        }
    }
    return dist;
}

// Entry value from the squared distance and the two point indices, one
// function per family (the tile generator picks the family once per CTA).
// Divisions by a kernel constant are multiplications by its reciprocal,
// computed once on the host (one rounding more than the reference's
// division: a relative change of at most |argument| ulp in an exponential,
// far below the 1e-13 the blocks are held to).
template <int FAM>
__device__ __forceinline__ double entry_fam(const DevKernel &K, double dist,
                                            long long ir, long long jc)
{
    if constexpr (FAM == FAM_EXP) {
        const double v = sqrt(dist) * K.inv_neg_beta;
        return v == 0.0 ? K.sigma + K.noise : K.sigma * exp(v);
    } else if constexpr (FAM == FAM_SQREXP) {
        const double v = dist * K.inv_neg_2beta2;
        return v == 0.0 ? K.sigma + K.noise : K.sigma * exp(v);
    } else if constexpr (FAM == FAM_MATERN || FAM == FAM_MATERN2) {
        const double x = sqrt(dist) * K.matern_scale;
        if (x == 0.0) return K.sigma + K.noise;
        // nu = 1/2, 3/2, 5/2: 2^(1-nu)/Gamma(nu) x^nu K_nu(x) is
        // exp(-x) times 1, 1 + x, 1 + x + x^2/3 (K_{n+1/2} is elementary)
        switch (K.matern_half) {
        case 1: return K.sigma * exp(-x);
        case 2: return K.sigma * ((1.0 + x) * exp(-x));
        case 3: return K.sigma * ((1.0 + x * (1.0 + x * (1.0 / 3.0))) * exp(-x));
        default:
            if (K.matern_tab != nullptr && x >= kMaternTabLo) {
                // e^-x underflows to zero long before 1024
                if (!(x < 1024.0)) return 0.0;
                return K.matern_coef * (exp(-x) * matern_tab_eval(K.matern_tab, x));
            }
            return K.matern_coef * pow(x, K.nu) * bessel_knu(K.nu, x);
        }
    } else if constexpr (FAM == FAM_COULOMB) {
        if (dist == 0.0) return K.zero_mode ? K.diag : 0.0;
        return __ddiv_rn(1.0, sqrt(dist));
    } else if constexpr (FAM == FAM_SIN || FAM == FAM_COS) {
        if (dist == 0.0) return K.diag;
        const double r = sqrt(dist);
        const double a = K.wave_k * r;
        return __ddiv_rn(FAM == FAM_SIN ? sin(a) : cos(a), r);
    } else {
        // the compactly supported bases amplify the rounding of x near
        // x = 1, so x is the reference's quotient here
        const double x = __ddiv_rn(sqrt(dist), K.rad);
        double v;
        switch (K.rbf_kind) {
        case 0: v = exp(-(x * x)); break;
        case 1: v = exp(-x); break;
        case 2: v = __ddiv_rn(1.0, 1.0 + x * x); break;
        case 3: v = __ddiv_rn(1.0, sqrt(1.0 + x * x)); break;
        case 4:
        case 5: v = exp(-x) + (1.0 + x); break;
        case 6: v = (x * x) * log(x); break;
        case 7: v = x > 1.0 ? 0.0 : pow(1.0 - x, 5.0); break;
        case 8: v = 1.0 + x * x; break;
        default: v = x > 1.0 ? 0.0 : pow(1.0 - x, 4.0) * (4.0 * x + 1.0);
        }
        // virus.c compares the truncated int point indices
        if (K.isreg && (int)ir == (int)jc) v += K.reg;
        return v;
    }
}

__device__ __forceinline__ double entry_from_dist(const DevKernel &K,
                                                  double dist, long long ir,
                                                  long long jc)
{
    switch (K.family) {
    case FAM_EXP: return entry_fam<FAM_EXP>(K, dist, ir, jc);
    case FAM_SQREXP: return entry_fam<FAM_SQREXP>(K, dist, ir, jc);
    case FAM_MATERN: return entry_fam<FAM_MATERN>(K, dist, ir, jc);
    case FAM_MATERN2: return entry_fam<FAM_MATERN2>(K, dist, ir, jc);
    case FAM_COULOMB: return entry_fam<FAM_COULOMB>(K, dist, ir, jc);
    case FAM_SIN: return entry_fam<FAM_SIN>(K, dist, ir, jc);
    case FAM_COS: return entry_fam<FAM_COS>(K, dist, ir, jc);
    case FAM_RBF: return entry_fam<FAM_RBF>(K, dist, ir, jc);
    }
    return 0.0;
}

// Entry (i, j) of the block whose rows are row_piv[row0 + i] and columns
// col_piv[col0 + j].
__device__ __forceinline__ double block_entry(const DevKernel &K,
                                              long long row0, long long col0,
                                              int i, int j)
{
    const long long ir = K.row_piv[row0 + i];
    const long long jc = K.col_piv[col0 + j];
    return entry_from_dist(K, sq_dist(K, ir, jc), ir, jc);
}

}  // namespace b200
