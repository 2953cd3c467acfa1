// FP32 rendering with forward tangents, the fast form behind the adjoint.
//
// Same work decomposition as render64.cu (pixel pass + per-level subsample
// warps over the device work queue), but per-pixel arithmetic is FP32 and
// every evaluation also returns the partial derivatives of the profile value
// with respect to profile coordinates and shape parameters.  For each
// radial profile and drawing pixel the pass stores NTAN sums
//   J0 = sum w f,   J1 = sum w df/dx',  J2 = sum w df/dy',
//   J3 = sum w df/dx' y',  J4 = sum w df/dy' x',  J5 = sum w df/dy' y',
//   J6..J8 = sum w df/d(shape parameter 1..3)
// over the pixel's quadrature points (w = sub-cell weights of the chosen
// subsampling).  The gradient of logL with respect to xcen, ycen, mag, ang,
// axrat and the shape parameters is a fixed linear combination of
// sum_pixels g(pixel) J_k(pixel), g being the adjoint of the convolution
// applied to dlogL/dmodel; the combination is done in FP64 on the host.
//
// FP64 is kept where FP32 would lose the answer:
//  - pixel and sub-cell coordinates relative to the profile centre are
//    formed in FP64 before rounding to FP32 (positions on a 2000-pixel
//    image would otherwise carry 1e-4 pixel errors), and sub-cell bounds
//    stay FP64 in the work queue (centre cells reach 8^-10 pixel);
//  - cells from recursion level 3 on (only the Sersic central cusp with
//    max_recursions = 10 gets there) are evaluated in FP64.

#include "common.cuh"
#include "conv.cuh"
#include "conv2.cuh"
#include "conv_tc.cuh"
#include "launch.h"
#include "like.cuh"

namespace pf {

// Value, position partials and parameter partials of one profile evaluation:
// s[0 .. shape_count(kind) - 1] are df/d(shape parameter k), s[shape_count]
// is df/dbox.
template <class T>
struct Tan {
	T f, fx, fy;
	T s[MAX_SHAPE + 1];
};

// FAST (FP32 only): the hardware approximations (ex2 / lg2 with one
// multiply; a few ulp, growing with |x| for the exponential) instead of
// CUDA's functions accurate to 1-2 ulp.  Used where only tangents are formed
// (the recomputing adjoint): their per-pixel errors of ~1e-6 stay an order
// below the gradient's accuracy bound, while the image values keep the
// accurate functions.
template <class T, bool FAST = false>
__device__ __forceinline__ T t_exp(T x)
{
	if constexpr (sizeof(T) == 8) return exp(x);
	else if constexpr (FAST) return __expf(x);
	else return expf(x);
}
template <class T, bool FAST = false>
__device__ __forceinline__ T t_log(T x)
{
	if constexpr (sizeof(T) == 8) return log(x);
	// (subnormal arguments keep the accurate function)
	else if constexpr (FAST) return x >= 1.17549435e-38f ? __logf(x) : logf(x);
	else return logf(x);
}
template <class T>
__device__ __forceinline__ T t_pow(T x, T y);
template <>
__device__ __forceinline__ float t_pow<float>(float x, float y) { return powf(x, y); }
template <>
__device__ __forceinline__ double t_pow<double>(double x, double y) { return pow(x, y); }
template <class T>
__device__ __forceinline__ T t_sqrt(T x);
template <>
__device__ __forceinline__ float t_sqrt<float>(float x) { return sqrtf(x); }
template <>
__device__ __forceinline__ double t_sqrt<double>(double x) { return sqrt(x); }

// a / b for divisors that vary from point to point.  The FP32 form takes the
// approximate quotient (reciprocal and one multiply, within 2 ulp; every
// divisor here is a normal number or guarded), a fraction of the IEEE
// division's instructions; the FP64 form keeps the IEEE quotient.  Per-profile
// constants (1/re, 1/n, ...) stay IEEE divisions: their rounding is the same
// at every pixel, so an approximate reciprocal would act as a shifted
// parameter, while the per-point errors average out over the image.
template <class T>
__device__ __forceinline__ T qdiv(T a, T b);
template <>
__device__ __forceinline__ float qdiv<float>(float a, float b) { return __fdividef(a, b); }
template <>
__device__ __forceinline__ double qdiv<double>(double a, double b) { return a / b; }

// x^y for x >= 0 given lx = ln x: exp(y lx), with pow's values at x = 0.
// The profiles need ln x for their partials anyway, so a power costs one
// exponential instead of pow's own logarithm and exponential.
template <class T, bool FAST = false>
__device__ __forceinline__ T pow_ln(T x, T lx, T y)
{
	if (x > T(0)) return t_exp<T, FAST>(y * lx);
	return y > T(0) ? T(0) : (y == T(0) ? T(1) : T(INFINITY));
}

// x^B for x >= 0 and a boxiness exponent B = 2 + box near 2, given lx = ln x:
// x^2 exp((B - 2) lx).  The exponential's argument stays small, so the
// rounding of lx is not amplified by |B lx| as in exp(B lx).
template <class T, bool FAST = false>
__device__ __forceinline__ T pow_box(T x, T lx, T B)
{
	if (x > T(0)) return x * x * t_exp<T, FAST>((B - T(2)) * lx);
	return pow_ln<T, FAST>(x, lx, B);
}

// ln x for x > 0, else 0 (every use multiplies it by a factor that is 0 there)
template <class T, bool FAST = false>
__device__ __forceinline__ T ln_pos(T x)
{
	return x > T(0) ? t_log<T, FAST>(x) : T(0);
}

// Sersic: f = exp(-bn (base^(1/(n B)) - 1)), base = |x/re|^B + |y/re|^B.
// Shape partials: s[0] = df/dre, s[1] = df/dnser (including dbn/dnser),
// s[2] = df/dbox.
template <class T, bool FAST = false, bool TAN = true>
__device__ __forceinline__ Tan<T> sersic_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t = {};
	const T B = (T)p.B, n = (T)p.nser, bn = (T)p.bn;
	const T ire = (T)p.k[0], in = (T)p.k[1], iB = (T)p.inv_B;
	const T u = fabs(xp) * ire, v = fabs(yp) * ire;
	T lu, lv, uB, vB;
	if (B == T(2)) {
		// ln u, ln v enter only the box partial here
		lu = TAN ? ln_pos<T, FAST>(u) : T(0);
		lv = TAN ? ln_pos<T, FAST>(v) : T(0);
		uB = u * u;
		vB = v * v;
	}
	else {
		lu = ln_pos<T, FAST>(u);
		lv = ln_pos<T, FAST>(v);
		uB = pow_box<T, FAST>(u, lu, B);
		vB = pow_box<T, FAST>(v, lv, B);
	}
	const T base = uB + vB;
	if (!(base > T(0))) {
		t.f = t_exp<T, FAST>(bn);
		return t;
	}
	const T inv_nB = (T)p.inv_nB;
	const T lnb = t_log<T, FAST>(base);
	const T rf = t_exp<T, FAST>(lnb * inv_nB);
	const T f = t_exp<T, FAST>(-bn * (rf - T(1)));
	t.f = f;
	if constexpr (!TAN) return t;
	const T dfdrf = -bn * f;
	const T h = dfdrf * rf * inv_nB;   // df/d ln(base)
	const T g = qdiv<T>(h, base);      // df/dbase
	// dbase/dx' = B uB / x' (= 2 x' / re^2 at B = 2)
	if (B == T(2)) {
		t.fx = g * T(2) * xp * ire * ire;
		t.fy = g * T(2) * yp * ire * ire;
	}
	else {
		t.fx = xp != T(0) ? g * B * qdiv<T>(uB, xp) : T(0);
		t.fy = yp != T(0) ? g * B * qdiv<T>(vB, yp) : T(0);
	}
	t.s[0] = -dfdrf * rf * in * ire;
	t.s[1] = -h * lnb * in - (rf - T(1)) * f * (T)p.dbn_dn;
	t.s[2] = h * (qdiv<T>(uB * lu + vB * lv, base) - lnb * iB);
	return t;
}

// Boxy radius r = (|x'|^B + |y'|^B)^(1/B) (radial.h:93-102) and its partials
// in x', y' and B.
template <class T, bool FAST = false, bool TAN = true>
__device__ __forceinline__ void boxy_radius(const FProfile &p, T xp, T yp, T &r, T &drdx, T &drdy, T &drdB)
{
	const T B = (T)p.B, ax = fabs(xp), ay = fabs(yp);
	drdx = drdy = drdB = T(0);
	if (B == T(2)) {
		const T S = xp * xp + yp * yp;
		r = t_sqrt<T>(S);
		if constexpr (!TAN) return;
		const T lx = ln_pos<T, FAST>(ax), ly = ln_pos<T, FAST>(ay);
		const T ir = r > T(0) ? qdiv<T>(T(1), r) : T(0);
		drdx = xp * ir;
		drdy = yp * ir;
		// r ((x'^2 ln|x'| + y'^2 ln|y'|) / (2 S) - ln S / 4)
		drdB = S > T(0) ? r * ((ax * ax * lx + ay * ay * ly) * ir * ir * T(0.5) - t_log<T, FAST>(S) * T(0.25)) : T(0);
	}
	else {
		const T lx = ln_pos<T, FAST>(ax), ly = ln_pos<T, FAST>(ay);
		const T xB = pow_box<T, FAST>(ax, lx, B), yB = pow_box<T, FAST>(ay, ly, B);
		const T S = xB + yB;
		const T iB = (T)p.inv_B;
		const T lS = ln_pos<T, FAST>(S);
		// S^(1/B) = sqrt(S) S^(1/B - 1/2), the second factor's exponent small
		r = S > T(0) ? t_sqrt<T>(S) * t_exp<T, FAST>(lS * (T)p.box_e) : T(0);
		if constexpr (!TAN) return;
		const T iS = S > T(0) ? qdiv<T>(T(1), S) : T(0);
		drdx = (r > T(0) && xp != T(0)) ? qdiv<T>(xB * iS * r, xp) : T(0);
		drdy = (r > T(0) && yp != T(0)) ? qdiv<T>(yB * iS * r, yp) : T(0);
		drdB = S > T(0) ? r * iB * ((xB * lx + yB * ly) * iS - lS * iB) : T(0);
	}
}

// Fills fx, fy and df/dbox (slot ns) from df/dr.
template <class T, bool FAST = false>
__device__ __forceinline__ void radial_chain(Tan<T> &t, T fr, T drdx, T drdy, T drdB, int ns)
{
	t.fx = fr * drdx;
	t.fy = fr * drdy;
	t.s[ns] = fr * drdB;
}

// Moffat: f = (1 + (r/rscale)^2)^-con.  s[0] = df/dfwhm, s[1] = df/dcon,
// s[2] = df/dbox.
template <class T, bool FAST = false, bool TAN = true>
__device__ __forceinline__ Tan<T> moffat_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t = {};
	const T irs = (T)p.k[0], con = (T)p.con;
	T r, drdx, drdy, drdB;
	boxy_radius<T, FAST, TAN>(p, xp, yp, r, drdx, drdy, drdB);
	const T rf = r * irs;
	const T q = T(1) + rf * rf;
	const T lq = t_log<T, FAST>(q);
	const T f = t_exp<T, FAST>(-con * lq);
	const T dfdrf = qdiv<T>(-T(2) * con * rf * f, q);
	t.f = f;
	if constexpr (!TAN) return t;
	radial_chain<T>(t, dfdrf * irs, drdx, drdy, drdB, 2);
	t.s[0] = dfdrf * (-rf) * (T)p.a;           // a holds 1/fwhm for Moffat
	t.s[1] = -lq * f + dfdrf * (-rf) * (T)p.b;  // b holds dln(rscale)/dcon
	return t;
}

// Ferrer: f = (1 - (r/rout)^(2-b))^a inside rout (ferrer.cpp:50-60).
// s[0] = df/drout, s[1] = df/da, s[2] = df/db, s[3] = df/dbox.
template <class T, bool FAST = false, bool TAN = true>
__device__ __forceinline__ Tan<T> ferrer_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t = {};
	T r, drdx, drdy, drdB;
	boxy_radius<T, FAST, TAN>(p, xp, yp, r, drdx, drdy, drdB);
	const T irout = (T)p.k[0], a = (T)p.a, e = T(2) - (T)p.b;
	const T rf = r * irout;
	if (!(rf < T(1))) return t;
	const T lrf = ln_pos<T, FAST>(rf);
	const T rfe = pow_ln<T, FAST>(rf, lrf, e);
	const T g = T(1) - rfe;
	const T lg = ln_pos<T, FAST>(g);
	const T f = pow_ln<T, FAST>(g, lg, a);
	t.f = f;
	if constexpr (!TAN) return t;
	if (!(g > T(0)) || !(r > T(0))) return t;
	const T ig = qdiv<T>(T(1), g);
	const T fr = -a * e * f * rfe * ig * qdiv<T>(T(1), r);
	radial_chain<T>(t, fr, drdx, drdy, drdB, 3);
	t.s[0] = -fr * r * irout;
	t.s[1] = f * lg;
	t.s[2] = a * f * rfe * lrf * ig;
	return t;
}

// King: f = ((1 + (r/rc)^2)^(-1/a) - (1 + (rt/rc)^2)^(-1/a))^a inside rt
// (king.cpp:51-59).  s[0] = df/drc, s[1] = df/drt, s[2] = df/da, s[3] = df/dbox.
template <class T, bool FAST = false, bool TAN = true>
__device__ __forceinline__ Tan<T> king_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t = {};
	T r, drdx, drdy, drdB;
	boxy_radius<T, FAST, TAN>(p, xp, yp, r, drdx, drdy, drdB);
	const T rc = (T)p.rc, rt = (T)p.rt, a = (T)p.a, kt = (T)p.king_t;
	if (!(r < rt)) return t;
	const T ia = (T)p.k[0], irc = (T)p.k[1];
	const T X = T(1) + (r * irc) * (r * irc);
	const T lX = t_log<T, FAST>(X);
	const T u = t_exp<T, FAST>(-lX * ia);
	const T D = u - kt;
	// D <= 0 only by rounding at r ~ rt, where pow keeps its own sign rules
	const T lD = ln_pos<T, FAST>(D);
	const T f = D > T(0) ? t_exp<T, FAST>(a * lD) : t_pow<T>(D, a);
	t.f = f;
	if constexpr (!TAN) return t;
	if (!(D > T(0))) return t;
	const T iX = qdiv<T>(T(1), X), iY = (T)p.k[2];
	const T k2 = T(2) * ia * irc * irc;
	const T du_dr = -k2 * r * u * iX;
	const T du_drc = k2 * r * r * u * irc * iX;
	const T dt_drc = k2 * rt * rt * kt * irc * iY;
	const T dt_drt = -k2 * rt * kt * iY;
	const T du_da = u * lX * ia * ia, dt_da = kt * (T)p.k[3] * ia * ia;
	const T c = a * f * qdiv<T>(T(1), D);
	radial_chain<T>(t, c * du_dr, drdx, drdy, drdB, 3);
	t.s[0] = c * (du_drc - dt_drc);
	t.s[1] = -c * dt_drt;
	t.s[2] = f * lD + c * (du_da - dt_da);
	return t;
}

// Broken exponential (brokenexponential.cpp:38-94): f = exp(-r/h1 +
// (1/h1 - 1/h2) base), base = log(1 + exp(a (r - rb)))/a, or r - rb where
// a (r - rb) >= 40.  s[0] = df/dh1, s[1] = df/dh2, s[2] = df/drb, s[3] = df/da,
// s[4] = df/dbox.
template <class T, bool FAST = false, bool TAN = true>
__device__ __forceinline__ Tan<T> brokenexp_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t = {};
	T r, drdx, drdy, drdB;
	boxy_radius<T, FAST, TAN>(p, xp, yp, r, drdx, drdy, drdB);
	const T a = (T)p.a, z = r - (T)p.rb;
	const T ih1 = (T)p.k[0], ih2 = (T)p.k[1], ia = (T)p.k[2];
	const T expo = ih1 - ih2;
	T base = z, dbase_dr = T(1), dbase_da = T(0);
	if (a * z < T(40)) {
		const T ez = t_exp<T, FAST>(a * z);
		base = t_log<T, FAST>(T(1) + ez) * ia;
		const T sig = qdiv<T>(ez, T(1) + ez);
		dbase_dr = sig;
		dbase_da = (z * sig - base) * ia;
	}
	const T f = t_exp<T, FAST>(-r * ih1 + expo * base);
	t.f = f;
	if constexpr (!TAN) return t;
	radial_chain<T>(t, f * (-ih1 + expo * dbase_dr), drdx, drdy, drdB, 4);
	t.s[0] = f * (r - base) * ih1 * ih1;
	t.s[1] = f * base * ih2 * ih2;
	t.s[2] = -f * expo * dbase_dr;
	t.s[3] = f * expo * dbase_da;
	return t;
}

// Core-Sersic (coresersic.cpp:51-59): f = (1 + (r/rb)^-a)^(b/a)
// exp(-bn ((r^a + rb^a)/re^a)^(1/(n a))).  s[0] = df/dre, s[1] = df/drb,
// s[2] = df/dnser (including dbn/dnser), s[3] = df/da, s[4] = df/db,
// s[5] = df/dbox.
template <class T, bool FAST = false, bool TAN = true>
__device__ __forceinline__ Tan<T> coresersic_tan(const FProfile &p, T xp, T yp)
{
	Tan<T> t = {};
	T r, drdx, drdy, drdB;
	boxy_radius<T, FAST, TAN>(p, xp, yp, r, drdx, drdy, drdB);
	const T a = (T)p.a, b = (T)p.b, rb = (T)p.rb, re = (T)p.re, n = (T)p.nser, bn = (T)p.bn;
	const T ia = (T)p.k[0], in = (T)p.k[1];
	const T lr = ln_pos<T, FAST>(r), lrb = (T)p.k[2], lre = (T)p.k[3];
	const T ra = pow_ln<T, FAST>(r, lr, a), rba = (T)p.k[4], irea = (T)p.k[5];
	// (r/rb)^-a, infinite at r = 0 for a > 0 as pow gives it
	const T rho = r > T(0) ? t_exp<T, FAST>(-a * (lr - lrb)) : pow_ln<T, FAST>(T(0), T(0), -a);
	const T A = T(1) + rho;
	const T Q = (ra + rba) * irea;
	const T lnQ = t_log<T, FAST>(Q);
	const T ina = (T)p.k[6];
	const T W = t_exp<T, FAST>(lnQ * ina);
	const T lnA = t_log<T, FAST>(A);
	const T ba = b * ia;
	const T f = t_exp<T, FAST>(ba == T(0) ? -bn * W : ba * lnA - bn * W);
	t.f = f;
	if constexpr (!TAN) return t;
	if (!(r > T(0)) || !(f > T(0))) return t;
	const T ir = qdiv<T>(T(1), r), irb = qdiv<T>(T(1), rb), iA = qdiv<T>(T(1), A), iQ = qdiv<T>(T(1), Q);
	const T dA_dr = -a * rho * ir, dA_drb = a * rho * irb, dA_da = -rho * (lr - lrb);
	const T dQ_dr = a * ra * ir * irea, dQ_drb = a * rba * irb * irea, dQ_dre = -a * Q / re;
	const T dlnQ_da = qdiv<T>(ra * lr + rba * lrb, ra + rba) - lre;
	const T wq = W * ina * iQ;  // dW/dQ
	const T dW_dn = -W * lnQ * ina * in;
	const T dW_da = W * ina * (dlnQ_da - lnQ * ia);
	radial_chain<T>(t, f * (ba * dA_dr * iA - bn * wq * dQ_dr), drdx, drdy, drdB, 5);
	t.s[0] = f * (-bn * wq * dQ_dre);
	t.s[1] = f * (ba * dA_drb * iA - bn * wq * dQ_drb);
	t.s[2] = f * (-(T)p.dbn_dn * W - bn * dW_dn);
	t.s[3] = f * (-(ba * ia) * lnA + ba * dA_da * iA - bn * dW_da);
	t.s[4] = f * lnA * ia;
	return t;
}

// AK (all kinds): false compiles only the Sersic and Moffat tangents, the
// kinds most models use, which keeps those kernels' code and registers as
// small as before the other kinds had gradients.
template <class T, bool AK, bool FAST = false, bool TAN = true>
__device__ __forceinline__ Tan<T> eval_tan(const FProfile &p, T xp, T yp)
{
	if (p.kind == PK_SERSIC) return sersic_tan<T, FAST, TAN>(p, xp, yp);
	if (p.kind == PK_MOFFAT) return moffat_tan<T, FAST, TAN>(p, xp, yp);
	if constexpr (AK) {
		switch (p.kind) {
		case PK_FERRER: return ferrer_tan<T, FAST, TAN>(p, xp, yp);
		case PK_CORESERSIC: return coresersic_tan<T, FAST, TAN>(p, xp, yp);
		case PK_KING: return king_tan<T, FAST, TAN>(p, xp, yp);
		case PK_BROKENEXP: return brokenexp_tan<T, FAST, TAN>(p, xp, yp);
		default: break;
		}
	}
	return Tan<T>{};
}

template <class T, bool AK, bool FAST = false>
__device__ __forceinline__ T eval_val(const FProfile &p, T xp, T yp)
{
	return eval_tan<T, AK, FAST, false>(p, xp, yp).f;
}

// Tangent slots the kernels of a kind set carry.
template <bool AK>
constexpr int ntk()
{
	return AK ? NTAN : NTAN_GEOM + 3;
}

// How one drawing pixel is integrated for one radial profile
// (radial.cpp:321-339): not at all (beyond rscale_max), by one evaluation,
// or by subsampling.  The forward pass and the recomputing adjoint must agree
// pixel for pixel, so this is written with round-to-nearest intrinsics,
// which no contraction or reassociation can change between kernels.
enum PixelDecision : int { PD_ZERO = 0, PD_DIRECT = 1, PD_SUBSAMPLE = 2 };

// The terms of a pixel column (centre x) in the rotated coordinates:
// dx cos(theta) and -dx sin(theta)/q, dx = x - xcen.  Kernels whose threads
// walk down a column form them once per profile.
struct ColumnTerms {
	float c, s;
};

__device__ __forceinline__ ColumnTerms column_terms(const FProfile &p, double x)
{
	const float dx = __double2float_rn(__dsub_rn(x, p.cx));
	return {__fmul_rn(dx, p.cos_ang), __fmul_rn(-dx, p.sin_q)};
}

__device__ __forceinline__ int pixel_decision32(const FProfile &p, ColumnTerms ct, double y, float &xp, float &yp)
{
	const float dy = __double2float_rn(__dsub_rn(y, p.cy));
	xp = __fadd_rn(ct.c, __fmul_rn(dy, p.sin_ang));
	yp = __fadd_rn(ct.s, __fmul_rn(dy, p.cos_q));
	const float r = __fsqrt_rn(__fadd_rn(__fmul_rn(xp, xp), __fmul_rn(yp, yp)));
	if (p.r_max > 0.f && r > p.r_max) return PD_ZERO;
	if (p.rough || r > p.r_switch) return PD_DIRECT;
	return PD_SUBSAMPLE;
}

__device__ __forceinline__ int pixel_decision32(const FProfile &p, double x, double y, float &xp, float &yp)
{
	return pixel_decision32(p, column_terms(p, x), y, xp, yp);
}

template <int NT>
__device__ __forceinline__ void tan_to_j(const Tan<float> &t, float xp, float yp, float w, float *j)
{
	j[0] += w * t.f;
	j[1] += w * t.fx;
	j[2] += w * t.fy;
	j[3] += w * t.fx * yp;
	j[4] += w * t.fy * xp;
	j[5] += w * t.fy * yp;
#pragma unroll
	for (int k = 0; k < NT - NTAN_GEOM; k++) j[NTAN_GEOM + k] += w * t.s[k];
}

template <class T>
__device__ __forceinline__ Tan<float> to_float(const Tan<T> &t)
{
	Tan<float> r;
	r.f = (float)t.f;
	r.fx = (float)t.fx;
	r.fy = (float)t.fy;
#pragma unroll
	for (int k = 0; k <= MAX_SHAPE; k++) r.s[k] = (float)t.s[k];
	return r;
}

// One thread per drawing pixel and per batch entry (blockIdx.z); prof_begin
// maps each batch entry to its range of FProfile records.  J: the tangents
// are written to the planes `jac` (false: values only, the tangent arithmetic
// is compiled out).  A profile whose rscale_max lies more than 2 px short of
// the block's nearest pixel centre is skipped for the whole block: the
// elliptical radius is never smaller than the Euclidean distance, so every
// pixel of the block would take the zero decision.  mask (optional, one
// drawing-size calculation mask for every batch entry): pixels where it is 0
// are not drawn by the radial and sky profiles (radial.cpp:306, sky.cpp:47-63).
// JT: element type of the tangent planes (float, or double where the cells
// of a subsampled pixel must be summed without FP32 cancellation).
// Pixel tiles of k_pixels32 (its block) and of k_jac_reduce: a profile whose
// r_max + 2 circle misses every pixel centre of a tile draws nothing there,
// and its tangent planes are neither written nor read on that tile.  Both
// kernels take this test, rounded alike (explicit FP32 operations, no
// contraction), so they skip the same tiles; FP32 rounding of coordinates
// below 2^13 px is far inside the 2 px margin, and subsampled cells lie
// inside r_switch < r_max, never on a skipped tile.
constexpr unsigned PIX_TILE_W = 32, PIX_TILE_H = 8;

// True when tile_culled keeps every tile of the drawing: every pixel centre
// lies within r_max + 1 of the profile centre (1 px inside the test's
// r_max + 2, far more than its FP32 rounding), or the profile has no r_max.
__device__ __forceinline__ bool tiles_all_reached(const FProfile &p, unsigned width, unsigned height, double sx,
                                                  double sy)
{
	if (!(p.r_max > 0.f)) return true;
	const double x0 = sx / 2., x1 = sx / 2. + (width - 1) * sy;  // x steps by sy, y by sx
	const double y0 = sy / 2., y1 = sy / 2. + (height - 1) * sx;
	const double fx = fmax(fabs(x0 - p.cx), fabs(x1 - p.cx)), fy = fmax(fabs(y0 - p.cy), fabs(y1 - p.cy));
	const double lim = (double)p.r_max + 1.0;
	return fx * fx + fy * fy <= lim * lim;
}

__device__ __forceinline__ bool tile_culled(const FProfile &p, unsigned tx0, unsigned ty0, unsigned width,
                                            unsigned height, double sx, double sy)
{
	if (!(p.r_max > 0.f)) return false;
	const float hx = __fmul_rn(__double2float_rn(sx), 0.5f), hy = __fmul_rn(__double2float_rn(sy), 0.5f);
	const float fx = __double2float_rn(sy), fy = __double2float_rn(sx);  // x steps by sy, y by sx
	const unsigned tx1 = min(tx0 + PIX_TILE_W - 1, width - 1), ty1 = min(ty0 + PIX_TILE_H - 1, height - 1);
	const float xlo = __fadd_rn(hx, __fmul_rn((float)tx0, fx)), xhi = __fadd_rn(hx, __fmul_rn((float)tx1, fx));
	const float ylo = __fadd_rn(hy, __fmul_rn((float)ty0, fy)), yhi = __fadd_rn(hy, __fmul_rn((float)ty1, fy));
	const float cx = __double2float_rn(p.cx), cy = __double2float_rn(p.cy);
	const float nx = __fsub_rn(fminf(fmaxf(cx, xlo), xhi), cx), ny = __fsub_rn(fminf(fmaxf(cy, ylo), yhi), cy);
	const float lim = __fadd_rn(p.r_max, 2.0f);
	return __fadd_rn(__fmul_rn(nx, nx), __fmul_rn(ny, ny)) > __fmul_rn(lim, lim);
}

template <bool AK, bool J, class JT>
__global__ void k_pixels32(const FProfile *__restrict__ profiles, const int *__restrict__ prof_begin,
                           unsigned width, unsigned height, double sx, double sy, float *__restrict__ img_conv,
                           float *__restrict__ img_plain, JT *__restrict__ jac, int nt, QueueSet q,
                           const uint8_t *__restrict__ mask, const int2 *__restrict__ extent)
{
	pdl_enter();
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned j = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (i >= width || j >= height) return;
	const size_t npix = (size_t)width * height;
	const uint32_t pix = i + j * width;
	if (extent && (i >= (unsigned)extent[b].x || j >= (unsigned)extent[b].y)) {
		// beyond what this entry's outputs read: zero images, no planes
		img_conv[(size_t)b * npix + pix] = 0.f;
		img_plain[(size_t)b * npix + pix] = 0.f;
		return;
	}
	const int p0 = prof_begin[b], p1 = prof_begin[b + 1];
	float acc[2] = {0.f, 0.f};
	const double half_xbin = sx / 2., half_ybin = sy / 2.;
	const double y = half_ybin + j * sx;
	const double x = half_xbin + i * sy;
	const unsigned tx0 = blockIdx.x * PIX_TILE_W, ty0 = blockIdx.y * PIX_TILE_H;
	const bool drawn = !mask || mask[pix];

	for (int pi = p0; pi < p1; pi++) {
		const FProfile &p = profiles[pi];
		if (p.kind == PK_SKY) {
			if (drawn) acc[p.target] += p.flux_scale;  // sky value is kept in flux_scale
			continue;
		}
		if (!is_radial_kind(p.kind)) continue;
		// block-uniform: nothing drawn, no tangent planes stored
		if (tile_culled(p, tx0, ty0, width, height, sx, sy)) continue;
		// planes of the kind's own tangents only (the reduction reads no more)
		const int nk = tangent_count(p.kind);
		if (!drawn) {
			if constexpr (J) {
				JT *jp = jac + (size_t)pi * nt * npix + pix;
				for (int k = 0; k < nk; k++) jp[(size_t)k * npix] = JT(0);
			}
			continue;
		}
		constexpr int NT = ntk<AK>();
		float jl[NT];
#pragma unroll
		for (int k = 0; k < NT; k++) jl[k] = 0.f;
		{
			float xp, yp;
			const int decision = pixel_decision32(p, x, y, xp, yp);
			if (decision == PD_ZERO) {
				// zero
			}
			else if (decision == PD_DIRECT) {
				if constexpr (J) {
					Tan<float> t = eval_tan<float, AK>(p, xp, yp);
					acc[p.target] += p.flux_scale * t.f;
					tan_to_j<NT>(t, xp, yp, 1.0f, jl);
				}
				else {
					acc[p.target] += p.flux_scale * eval_val<float, AK>(p, xp, yp);
				}
			}
			else {
				unsigned res = p.resolution, max_rec = p.max_rec;
				if (p.centre_override && fabs(x - p.cx) < p.img_sx && fabs(y - p.cy) < p.img_sy) {
					res = 8;
					max_rec = 10;
				}
				SubItem it;
				const double ddx = x - p.cx, ddy = y - p.cy;
				it.x0 = ddx - half_xbin;
				it.x1 = ddx + half_xbin;
				it.y0 = ddy - half_ybin;
				it.y1 = ddy + half_ybin;
				it.weight = 1.0 / (res * res);
				it.pixel = pix + (uint32_t)(b * npix);
				it.profile = (uint16_t)pi;
				it.res = (uint8_t)res;
				it.max_rec = (uint8_t)max_rec;
				queue_push(q, 0, it);
				note_max_res(q, res);
			}
		}
		if constexpr (J) {
			JT *jp = jac + (size_t)pi * nt * npix + pix;
#pragma unroll
			for (int k = 0; k < NT; k++)
				if (k < nk) jp[(size_t)k * npix] = (JT)jl[k];
		}
	}
	img_conv[(size_t)b * npix + pix] = acc[0];
	img_plain[(size_t)b * npix + pix] = acc[1];
}

// The render without tangent planes, for models with many profiles: each
// block first lists, in profile order, the profiles that reach its tile (the
// sky, and radial profiles not skipped by k_pixels32's block test, evaluated
// the same way over the tile), then every pixel loops over that list only.
// Profiles are listed 256 at a time, one per thread, with an ordered
// compaction (warp ballots), so each pixel adds the same terms in the same
// order as k_pixels32 without planes: the images are the same bit for bit.
// Each thread takes two pixels, rows LISTED_ROWS apart, so one load of a
// profile's scalars serves both.
constexpr int LISTED_ROWS = 8;  // thread rows of a block; the tile is 32 x 2*LISTED_ROWS

template <bool AK>
__device__ __forceinline__ void listed_pixel(const FProfile &p, int pi, double x, double y, double half_xbin,
                                             double half_ybin, uint32_t pix, int b, size_t npix, float *acc,
                                             const QueueSet &q)
{
	if (p.kind == PK_SKY) {
		acc[p.target] += p.flux_scale;  // sky value is kept in flux_scale
		return;
	}
	float xp, yp;
	// (forming the column terms once per profile for both rows took this
	// kernel from 48 to 56 registers and one CTA per SM, a net loss)
	const int decision = pixel_decision32(p, x, y, xp, yp);
	if (decision == PD_DIRECT) {
		acc[p.target] += p.flux_scale * eval_val<float, AK>(p, xp, yp);
	}
	else if (decision == PD_SUBSAMPLE) {
		unsigned res = p.resolution, max_rec = p.max_rec;
		if (p.centre_override && fabs(x - p.cx) < p.img_sx && fabs(y - p.cy) < p.img_sy) {
			res = 8;
			max_rec = 10;
		}
		SubItem it;
		const double ddx = x - p.cx, ddy = y - p.cy;
		it.x0 = ddx - half_xbin;
		it.x1 = ddx + half_xbin;
		it.y0 = ddy - half_ybin;
		it.y1 = ddy + half_ybin;
		it.weight = 1.0 / (res * res);
		it.pixel = pix + (uint32_t)(b * npix);
		it.profile = (uint16_t)pi;
		it.res = (uint8_t)res;
		it.max_rec = (uint8_t)max_rec;
		queue_push(q, 0, it);
		note_max_res(q, res);
	}
}

template <bool AK>
__global__ void __launch_bounds__(256) k_pixels32_listed(const FProfile *__restrict__ profiles,
                                                         const int *__restrict__ prof_begin, unsigned width,
                                                         unsigned height, double sx, double sy,
                                                         float *__restrict__ img_conv, float *__restrict__ img_plain,
                                                         QueueSet q, const uint8_t *__restrict__ mask)
{
	pdl_enter();
	__shared__ int s_list[256];
	__shared__ int s_count[8];
	const int lane = threadIdx.x, wid = threadIdx.y, tid = wid * 32 + lane;
	const unsigned i = blockIdx.x * 32 + threadIdx.x;
	const unsigned ty0 = blockIdx.y * (2 * LISTED_ROWS);
	const unsigned j[2] = {ty0 + threadIdx.y, ty0 + LISTED_ROWS + threadIdx.y};
	const int b = blockIdx.z;
	const size_t npix = (size_t)width * height;
	const int p0 = prof_begin[b], p1 = prof_begin[b + 1];
	const double half_xbin = sx / 2., half_ybin = sy / 2.;
	const double x = half_xbin + i * sy;
	bool inside[2], drawn[2];
	uint32_t pix[2];
	double y[2];
	float acc[2][2] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
	for (int r = 0; r < 2; r++) {
		inside[r] = i < width && j[r] < height;
		pix[r] = inside[r] ? i + j[r] * width : 0;
		y[r] = half_ybin + j[r] * sx;
		drawn[r] = inside[r] && (!mask || mask[pix[r]]);
	}
	// pixel centres of this tile (same expressions as x and y)
	const unsigned tx0 = blockIdx.x * 32;
	const unsigned tx1 = min(tx0 + 31, width - 1), ty1 = min(ty0 + 2 * LISTED_ROWS - 1, height - 1);
	const double xlo = half_xbin + tx0 * sy, xhi = half_xbin + tx1 * sy;
	const double ylo = half_ybin + ty0 * sx, yhi = half_ybin + ty1 * sx;

	for (int base = p0; base < p1; base += 256) {
		bool keep = false;
		if (base + tid < p1) {
			const FProfile &p = profiles[base + tid];
			if (p.kind == PK_SKY) {
				keep = true;
			}
			else if (is_radial_kind(p.kind)) {
				keep = true;
				if (p.r_max > 0.f) {
					const double nx = fmin(fmax(p.cx, xlo), xhi) - p.cx, ny = fmin(fmax(p.cy, ylo), yhi) - p.cy;
					const double lim = (double)p.r_max + 2.0;
					keep = !(nx * nx + ny * ny > lim * lim);
				}
			}
		}
		const unsigned ballot = __ballot_sync(0xffffffffu, keep);
		if (lane == 0) s_count[wid] = __popc(ballot);
		__syncthreads();
		int before = 0, total = 0;
#pragma unroll
		for (int w = 0; w < 8; w++) {
			before += w < wid ? s_count[w] : 0;
			total += s_count[w];
		}
		if (keep) s_list[before + __popc(ballot & ((1u << lane) - 1u))] = base + tid;
		__syncthreads();
		if (drawn[0] || drawn[1]) {
			for (int k = 0; k < total; k++) {
				const int pi = s_list[k];
				const FProfile &p = profiles[pi];
#pragma unroll
				for (int r = 0; r < 2; r++)
					if (drawn[r]) listed_pixel<AK>(p, pi, x, y[r], half_xbin, half_ybin, pix[r], b, npix, acc[r], q);
			}
		}
		__syncthreads();  // the next round rewrites s_list and s_count
	}
#pragma unroll
	for (int r = 0; r < 2; r++)
		if (inside[r]) {
			img_conv[(size_t)b * npix + pix[r]] = acc[r][0];
			img_plain[(size_t)b * npix + pix[r]] = acc[r][1];
		}
}

// k / res == (k * div_magic(res)) >> 16 for every sub-point index k < 256
// and resolution 1 <= res <= 16: the magic ceil(2^16 / res) exceeds 2^16 / res
// by less than 1, so the product overshoots k / res by less than 256 / 2^16,
// short of the 1 / res gap to the next integer.
__device__ __forceinline__ unsigned div_magic(unsigned res)
{
	return (65536u + res - 1) / res;
}

// Sub-points [base0, base1) of an item (multiples of 32), one per lane and
// chunk.
template <class T, bool AK, bool J>
__device__ __forceinline__ void level_points(const FProfile &p, const SubItem &it, int level, const double *s_xy,
                                             int lane, const QueueSet &q, float *sums, uint32_t *mask_out,
                                             unsigned base0, unsigned base1)
{
	const unsigned res = it.res;
	const double xbin = (it.x1 - it.x0) / res, ybin = (it.y1 - it.y0) / res;
	const double half_xbin = xbin / 2., half_ybin = ybin / 2.;
	const bool recurse = res > 1 && (unsigned)level < it.max_rec;
	const T adyp = fabs((T)(-xbin * (double)p.sin_q + ybin * (double)p.cos_q));
	const T cos_a = (T)p.cos_ang, sin_a = (T)p.sin_ang, cos_q = (T)p.cos_q, sin_q = (T)p.sin_q;
	const unsigned nsub = res * res, mres = div_magic(res);
	// sub-points in warp-wide chunks of 32 so each chunk's accept bits can be
	// gathered with one ballot (mask_out: the item's 8 words, or null)
	for (unsigned base = base0; base < base1 && base < nsub; base += 32) {
		const unsigned k = base + lane;
		bool accepted = false;
		if (k < nsub) {
			unsigned ii = (k * mres) >> 16, jj = k - ii * res;
			const double x = s_xy[ii], y = s_xy[16 + jj];
			const T dx = (T)x, dy = (T)y;
			const T xp = dx * cos_a + dy * sin_a;
			const T yp = -dx * sin_q + dy * cos_q;
			// the test point is evaluated beside the sub-point (independent
			// chains the scheduler can interleave)
			Tan<T> t = eval_tan<T, AK>(p, xp, yp);
			const T testval = recurse ? eval_val<T, AK>(p, fabs(xp), fabs(yp) + adyp) : T(0);
			accepted = true;
			if (recurse) {
				if (fabs(testval - t.f) > (T)p.acc * t.f) {
					accepted = false;
					SubItem c;
					c.x0 = x - half_xbin;
					c.x1 = x + half_xbin;
					c.y0 = y - half_ybin;
					c.y1 = y + half_ybin;
					c.weight = it.weight / nsub;
					c.pixel = it.pixel;
					c.profile = it.profile;
					c.res = it.res;
					c.max_rec = it.max_rec;
					if ((uint32_t)level + 1 < q.levels) queue_push(q, level + 1, c);
					else atomicOr(q.overflow, 2u);
				}
			}
			if (accepted) {
				if constexpr (J) tan_to_j<ntk<AK>()>(to_float<T>(t), (float)xp, (float)yp, 1.0f, sums);
				else sums[0] += (float)t.f;
			}
		}
		const unsigned bits = __ballot_sync(0xffffffffu, accepted);
		if (mask_out && lane == 0) mask_out[base >> 5] = bits;
	}
}

// Adjoint of one item with its frozen decisions: the tangents of the
// sub-points the forward pass accepted (mask bit set), summed.
template <class T, bool AK>
__device__ __forceinline__ void adjoint_points(const FProfile &p, const SubItem &it, const double *s_xy, int lane,
                                               const uint32_t *mask, float *sums)
{
	const unsigned res = it.res;
	const T cos_a = (T)p.cos_ang, sin_a = (T)p.sin_ang, cos_q = (T)p.cos_q, sin_q = (T)p.sin_q;
	const unsigned nsub = res * res, mres = div_magic(res);
	for (unsigned k = lane; k < nsub; k += 32) {
		if (!((mask[k >> 5] >> (k & 31)) & 1u)) continue;
		unsigned ii = (k * mres) >> 16, jj = k - ii * res;
		const double x = s_xy[ii], y = s_xy[16 + jj];
		const T dx = (T)x, dy = (T)y;
		const T xp = dx * cos_a + dy * sin_a;
		const T yp = -dx * sin_q + dy * cos_q;
		Tan<T> t = eval_tan<T, AK, true>(p, xp, yp);  // tangents only: fast functions
		tan_to_j<ntk<AK>()>(to_float<T>(t), (float)xp, (float)yp, 1.0f, sums);
	}
}

// Sub-points [base0, base1) of one SubItem integrated by one warp (s_xy:
// this warp's 32 doubles); FP64 sub-points from level 3 on (the Sersic cusp).
// J: tangents are accumulated into the planes `jac` (false: values only, the
// tangent arithmetic is compiled out).
template <bool Deep, bool AK, bool J, class JT>
__device__ __forceinline__ void level32_item(const FProfile *__restrict__ profiles, const SubItem &it, int level,
                                             unsigned npix, float *__restrict__ img_conv,
                                             float *__restrict__ img_plain, JT *__restrict__ jac, int nt,
                                             const QueueSet &q, double *s_xy, int lane, uint32_t *mask_out,
                                             unsigned base0, unsigned base1)
{
	const FProfile &p = profiles[it.profile];
	const unsigned res = it.res;
	const double half_xbin = (it.x1 - it.x0) / res / 2., half_ybin = (it.y1 - it.y0) / res / 2.;
	if (lane < 16) {
		if (lane < (int)res) s_xy[lane] = it.x0 + (2 * lane + 1) * half_xbin;
	}
	else if (lane - 16 < (int)res) {
		s_xy[lane] = it.y0 + (2 * (lane - 16) + 1) * half_ybin;
	}
	__syncwarp();
	constexpr int NT = ntk<AK>();
	float sums[NT];
#pragma unroll
	for (int k = 0; k < NT; k++) sums[k] = 0.f;
	if constexpr (Deep) level_points<double, AK, J>(p, it, level, s_xy, lane, q, sums, mask_out, base0, base1);
	else level_points<float, AK, J>(p, it, level, s_xy, lane, q, sums, mask_out, base0, base1);
	float *img = p.target == 0 ? img_conv : img_plain;
	if constexpr (J) {
		// lane 2m ends with the cell's sum of tangent m (m = 0: the value) and
		// adds it to its plane
		const float tot = warp_sums_spread<NT>(sums, lane);
		const int m = lane >> 1, nk = tangent_count(p.kind);
		if (lane == 0) atomicAdd(&img[it.pixel], (float)(p.flux_scale64 * it.weight * (double)tot));
		if ((lane & 1) == 0 && m < nk) {
			const uint32_t b = it.pixel / npix, pix = it.pixel - b * npix;
			JT *jp = jac + (size_t)it.profile * nt * npix + pix;
			// FP32 planes: the FP32 product; FP64 planes: the cell's sums
			// enter at full precision (a pixel's cells can cancel)
			const JT w = sizeof(JT) == 8 ? (JT)it.weight : (JT)(float)it.weight;
			atomicAdd(&jp[(size_t)m * npix], w * (JT)tot);
		}
	}
	else {
		const float tot = warp_sum(sums[0]);
		if (lane == 0) atomicAdd(&img[it.pixel], (float)(p.flux_scale64 * it.weight * (double)tot));
	}
	__syncwarp();
}

// Deep: FP64 sub-points (levels >= 3, the Sersic cusp).
template <bool AK, bool J, bool Deep, class JT>
__global__ void __launch_bounds__(256, Deep ? 2 : (AK ? 3 : 4)) k_level32(const FProfile *__restrict__ profiles, int level, unsigned npix,
                                                 float *__restrict__ img_conv, float *__restrict__ img_plain,
                                                 JT *__restrict__ jac, int nt, QueueSet q)
{
	pdl_enter();
	__shared__ double s_xy[8][32];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint32_t n = min(q.counts[level], q.cap[level]);
	const SubItem *items = q.items + q.off[level];
	const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
	// Fewer items than warps (a single image): one warp per (item, chunk of
	// 32 sub-points), so an item's chunks run side by side; otherwise one warp
	// per item.
	uint32_t cpi = 1;
	if (n < nwarps) {
		uint32_t maxres = q.maxres ? *q.maxres : 16u;
		if (maxres == 0 || maxres > 16) maxres = 16;
		cpi = (maxres * maxres + 31) / 32;
	}
	const uint32_t total = n * cpi;
	// kind-grouped order when the items were grouped (models with every kind)
	const uint32_t *perm = (!Deep && q.perm) ? q.perm + q.off[level] : nullptr;
	for (uint32_t w = blockIdx.x * (blockDim.x >> 5) + wib; w < total; w += nwarps) {
		const uint32_t slot = w / cpi, chunk = w - slot * cpi;
		const uint32_t item = perm ? perm[slot] : slot;
		const SubItem it = items[item];
		const unsigned base0 = cpi == 1 ? 0u : chunk * 32, base1 = cpi == 1 ? 256u : base0 + 32;
		if (base0 >= (unsigned)it.res * it.res) continue;
		level32_item<Deep, AK, J, JT>(profiles, it, level, npix, img_conv, img_plain, jac, nt, q, s_xy[wib], lane,
		                    q.masks ? q.masks + ((size_t)q.off[level] + item) * MASK_WORDS : nullptr, base0,
		                    base1);
	}
}

// Levels first..levels-1 in one CTA.  Only the Sersic central cusp
// (max_recursions = 10) reaches these levels, a few hundred cells per level
// at most, so one block walks them in order; __syncthreads separates the
// levels, which makes every push of level L visible before level L+1 is read.
template <bool AK, bool J, class JT>
__global__ void __launch_bounds__(512) k_deep_levels32(const FProfile *__restrict__ profiles, int first, int levels,
                                                        unsigned npix, float *__restrict__ img_conv,
                                                        float *__restrict__ img_plain, JT *__restrict__ jac,
                                                        int nt, QueueSet q)
{
	pdl_enter();
	__shared__ double s_xy[16][32];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint32_t nwarps = blockDim.x >> 5;
	for (int level = first; level < levels; level++) {
		__syncthreads();
		const uint32_t n = min(*(volatile uint32_t *)&q.counts[level], q.cap[level]);
		const SubItem *items = q.items + q.off[level];
		for (uint32_t w = wib; w < n; w += nwarps)
			level32_item<true, AK, J, JT>(profiles, items[w], level, npix, img_conv, img_plain, jac, nt, q, s_xy[wib], lane,
			                   q.masks ? q.masks + ((size_t)q.off[level] + w) * MASK_WORDS : nullptr, 0, 256);
	}
}

// ---------------------------------------------------------------------------
// Recomputing adjoint (no stored tangent planes): used when the planes would
// not fit, e.g. hundreds of profiles on a large field.  The forward pass
// rendered values only and recorded each queued cell's accepted sub-points;
// these kernels recompute the tangents against the known seed g.
// ---------------------------------------------------------------------------

// Directly evaluated pixels, one profile per blockIdx.z, 64 x 32 pixel tiles.
// A tile whose nearest pixel centre is farther than rscale_max (+2 px) from
// the profile centre is skipped: the elliptical radius is never smaller than
// the Euclidean distance, so such pixels were zeroed by the forward pass.
template <bool AK>
__global__ void __launch_bounds__(256) k_adjoint_pixels32(const FProfile *__restrict__ profiles,
                                                          const int *__restrict__ prof_batch, unsigned width,
                                                          unsigned height, double sx, double sy,
                                                          const float *__restrict__ g_conv,
                                                          const float *__restrict__ g_plain, double *__restrict__ T,
                                                          const uint8_t *__restrict__ mask)
{
	pdl_enter();
	const int pi = blockIdx.z;
	const FProfile &p = profiles[pi];
	if (!is_radial_kind(p.kind)) return;
	const unsigned tx0 = blockIdx.x * 64, ty0 = blockIdx.y * 32;
	const double half_xbin = sx / 2., half_ybin = sy / 2.;
	if (p.r_max > 0.f) {
		const unsigned tx1 = min(tx0 + 63, width - 1), ty1 = min(ty0 + 31, height - 1);
		const double xlo = half_xbin + tx0 * sy, xhi = half_xbin + tx1 * sy;
		const double ylo = half_ybin + ty0 * sx, yhi = half_ybin + ty1 * sx;
		const double nx = fmin(fmax(p.cx, xlo), xhi) - p.cx, ny = fmin(fmax(p.cy, ylo), yhi) - p.cy;
		if (sqrt(nx * nx + ny * ny) > (double)p.r_max + 2.0) return;
	}
	const size_t npix = (size_t)width * height;
	const float *g = (p.target == 0 ? g_conv : g_plain) + (size_t)prof_batch[pi] * npix;
	constexpr int NT = ntk<AK>();
	float acc[NT];
#pragma unroll
	for (int k = 0; k < NT; k++) acc[k] = 0.f;
	const unsigned i = tx0 + (threadIdx.x & 63);
	for (unsigned r = threadIdx.x >> 6; r < 32; r += 4) {
		const unsigned j = ty0 + r;
		if (i >= width || j >= height) continue;
		if (mask && !mask[i + (size_t)j * width]) continue;  // not drawn by the forward pass
		const float gv = g[i + (size_t)j * width];
		if (gv == 0.f) continue;
		const double y = half_ybin + j * sx, x = half_xbin + i * sy;
		float xp, yp;
		if (pixel_decision32(p, x, y, xp, yp) != PD_DIRECT) continue;
		Tan<float> t = eval_tan<float, AK, true>(p, xp, yp);
		tan_to_j<NT>(t, xp, yp, gv, acc);
	}
	__shared__ double s_red[NT][8];
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	{
		// lane 2m ends with the warp's sum of tangent m
		double a[NT];
#pragma unroll
		for (int k = 0; k < NT; k++) a[k] = (double)acc[k];
		const double v = warp_sums_spread<NT>(a, lane);
		if ((lane & 1) == 0 && (lane >> 1) < NT) s_red[lane >> 1][wid] = v;
	}
	__syncthreads();
	if (threadIdx.x < NT) {
		double v = 0;
		for (int w = 0; w < 8; w++) v += s_red[threadIdx.x][w];
		if (v != 0.0) atomicAdd(&T[(size_t)pi * NTAN + threadIdx.x], v);
	}
}

// The same for models with many profiles per batch entry: one block per
// 64 x 32 tile and batch entry lists the profiles whose rscale_max (+2 px)
// reaches the tile (the test above), then takes them one after another.  A
// block per (tile, profile) left most blocks with nothing to do but that
// test: on a large field the launch of the culled blocks cost more than the
// test itself.  (T is added atomically either way, in no fixed order.)
template <bool AK>
__global__ void __launch_bounds__(256, AK ? 3 : 5) k_adjoint_pixels32_listed(const FProfile *__restrict__ profiles,
                                                                 const int *__restrict__ prof_begin, unsigned width,
                                                                 unsigned height, double sx, double sy,
                                                                 const float *__restrict__ g_conv,
                                                                 const float *__restrict__ g_plain,
                                                                 double *__restrict__ T,
                                                                 const uint8_t *__restrict__ mask)
{
	pdl_enter();
	constexpr int NT = ntk<AK>();
	__shared__ int s_list[256];
	__shared__ int s_count;
	__shared__ double s_red[NT][8];
	const int b = blockIdx.z;
	const unsigned tx0 = blockIdx.x * 64, ty0 = blockIdx.y * 32;
	const double half_xbin = sx / 2., half_ybin = sy / 2.;
	const unsigned tx1 = min(tx0 + 63, width - 1), ty1 = min(ty0 + 31, height - 1);
	const double xlo = half_xbin + tx0 * sy, xhi = half_xbin + tx1 * sy;
	const double ylo = half_ybin + ty0 * sx, yhi = half_ybin + ty1 * sx;
	const size_t npix = (size_t)width * height;
	const int p0 = prof_begin[b], p1 = prof_begin[b + 1];
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
	const unsigned i = tx0 + (threadIdx.x & 63);
	for (int base = p0; base < p1; base += 256) {
		if (threadIdx.x == 0) s_count = 0;
		__syncthreads();
		if (base + (int)threadIdx.x < p1) {
			const int pi = base + threadIdx.x;
			const FProfile &p = profiles[pi];
			bool keep = is_radial_kind(p.kind);
			if (keep && p.r_max > 0.f) {
				const double nx = fmin(fmax(p.cx, xlo), xhi) - p.cx, ny = fmin(fmax(p.cy, ylo), yhi) - p.cy;
				keep = !(sqrt(nx * nx + ny * ny) > (double)p.r_max + 2.0);
			}
			if (keep) s_list[atomicAdd(&s_count, 1)] = pi;
		}
		__syncthreads();
		const int n = s_count;
		for (int k = 0; k < n; k++) {
			const int pi = s_list[k];
			const FProfile &p = profiles[pi];
			const float *g = (p.target == 0 ? g_conv : g_plain) + (size_t)b * npix;
			float acc[NT];
#pragma unroll
			for (int t = 0; t < NT; t++) acc[t] = 0.f;
			const ColumnTerms ct = column_terms(p, half_xbin + i * sy);  // the thread's column
			for (unsigned r = threadIdx.x >> 6; r < 32; r += 4) {
				const unsigned j = ty0 + r;
				if (i >= width || j >= height) continue;
				if (mask && !mask[i + (size_t)j * width]) continue;  // not drawn by the forward pass
				const float gv = g[i + (size_t)j * width];
				if (gv == 0.f) continue;
				const double y = half_ybin + j * sx;
				float xp, yp;
				if (pixel_decision32(p, ct, y, xp, yp) != PD_DIRECT) continue;
				Tan<float> t = eval_tan<float, AK, true>(p, xp, yp);
				tan_to_j<NT>(t, xp, yp, gv, acc);
			}
			{
				// lane 2m ends with the warp's sum of tangent m
				double a[NT];
#pragma unroll
				for (int t = 0; t < NT; t++) a[t] = (double)acc[t];
				const double v = warp_sums_spread<NT>(a, lane);
				if ((lane & 1) == 0 && (lane >> 1) < NT) s_red[lane >> 1][wid] = v;
			}
			__syncthreads();
			if (threadIdx.x < NT) {
				double v = 0;
				for (int w = 0; w < 8; w++) v += s_red[threadIdx.x][w];
				if (v != 0.0) atomicAdd(&T[(size_t)pi * NTAN + threadIdx.x], v);
			}
			__syncthreads();  // s_red is rewritten for the next profile
		}
	}
}

// Every queued cell of every level, one warp per cell: the tangents of the
// accepted sub-points, times the cell weight and g(pixel).
template <bool AK>
__global__ void __launch_bounds__(256) k_adjoint_items32(const FProfile *__restrict__ profiles, int levels,
                                                         const float *__restrict__ g_conv,
                                                         const float *__restrict__ g_plain, QueueSet q,
                                                         double *__restrict__ T)
{
	pdl_enter();
	__shared__ double s_xy[8][32];
	const int lane = threadIdx.x & 31;
	const int wib = threadIdx.x >> 5;
	const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
	const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + wib;
	for (int level = 0; level < levels; level++) {
		const uint32_t n = min(q.counts[level], q.cap[level]);
		const SubItem *items = q.items + q.off[level];
		for (uint32_t w = gw; w < n; w += nwarps) {
			const SubItem it = items[w];
			const FProfile &p = profiles[it.profile];
			const unsigned res = it.res;
			const double half_xbin = (it.x1 - it.x0) / res / 2., half_ybin = (it.y1 - it.y0) / res / 2.;
			if (lane < 16) {
				if (lane < (int)res) s_xy[wib][lane] = it.x0 + (2 * lane + 1) * half_xbin;
			}
			else if (lane - 16 < (int)res) {
				s_xy[wib][lane] = it.y0 + (2 * (lane - 16) + 1) * half_ybin;
			}
			__syncwarp();
			const uint32_t *mask = q.masks + ((size_t)q.off[level] + w) * MASK_WORDS;
			constexpr int NT = ntk<AK>();
			float sums[NT];
#pragma unroll
			for (int k = 0; k < NT; k++) sums[k] = 0.f;
			if (level >= 3) adjoint_points<double, AK>(p, it, s_xy[wib], lane, mask, sums);
			else adjoint_points<float, AK>(p, it, s_xy[wib], lane, mask, sums);
			{
				// lane 2m ends with the cell's sum of tangent m and adds it to T
				const float tot = warp_sums_spread<NT>(sums, lane);
				const int m = lane >> 1;
				if ((lane & 1) == 0 && m < NT) {
					const float gv = (p.target == 0 ? g_conv : g_plain)[it.pixel];
					const double coef = (double)gv * it.weight;
					if (coef != 0.0) atomicAdd(&T[(size_t)it.profile * NTAN + m], coef * (double)tot);
				}
			}
			__syncwarp();
		}
	}
}

cudaError_t launch_adjoint_recompute(const FProfile *profiles, const int *prof_batch, const int *prof_begin,
                                     int batch, int n_profiles, unsigned width, unsigned height, double sx, double sy,
                                     const float *g_conv, const float *g_plain, int levels, bool all_kinds,
                                     const QueueSet &q, double *T, cudaStream_t s, const uint8_t *mask)
{
	cudaError_t e;
	auto ki = all_kinds ? k_adjoint_items32<true> : k_adjoint_items32<false>;
	if (n_profiles >= ADJOINT_LIST_MIN_PROFILES * batch) {
		dim3 grid((width + 63) / 64, (height + 31) / 32, batch);
		auto kl = all_kinds ? k_adjoint_pixels32_listed<true> : k_adjoint_pixels32_listed<false>;
		e = launch_pdl(kl, grid, dim3(256), 0, s, profiles, prof_begin, width, height, sx, sy, g_conv, g_plain, T, mask);
	}
	else {
		dim3 grid((width + 63) / 64, (height + 31) / 32, n_profiles);
		auto kp = all_kinds ? k_adjoint_pixels32<true> : k_adjoint_pixels32<false>;
		e = launch_pdl(kp, grid, dim3(256), 0, s, profiles, prof_batch, width, height, sx, sy, g_conv, g_plain, T,
		               mask);
	}
	if (e == cudaSuccess) e = launch_pdl(ki, dim3(148 * 8), dim3(256), 0, s, profiles, levels, g_conv, g_plain, q, T);
	note_launches(2);
	return e;
}

// The batch gradient step: logL and d logL / d parameter of every
// (proposal, parameter) from the tangent reductions T.  k_batch_gradient runs
// it as its own launch; k_jac_reduce can run it in the block that completes
// the last profile (ticket: one zero-initialised word over all profiles,
// left at zero), which saves the launch when the batch is small.

// The inputs of gradient-step entry t that do not depend on T (t < batch
// also covers logL of proposal t; thread t < ctrl_words one control word,
// thread 0 the completion word).  Loaded ahead of the tickets that decide
// which block runs the step, so that the step itself waits on T and the
// profile records only.
struct GradPre {
	double ll = 0;
	int inv_t = 0, inv_b = 0, pi = 0, code = 0;
	uint32_t ctrl = 0;
	unsigned seq = 0;
};

__device__ __forceinline__ GradPre grad_prefetch(const GradStepArgs &g, int t)
{
	GradPre f;
	if (t < g.batch) {
		f.inv_t = __ldcg(g.invalid + t);
		f.ll = __ldcg(g.ll + t);
	}
	if (t < g.batch * g.nrefs) {
		const int b = t / g.nrefs, r = t - b * g.nrefs;
		f.pi = b * g.nprof + __ldcg(g.ref_profile + r);
		f.code = __ldcg(g.ref_code + r);
		f.inv_b = __ldcg(g.invalid + b);
	}
	if (g.ctrl_out && t < g.ctrl_words) f.ctrl = __ldcg(g.ctrl_in + t);
	if (g.seq_out && t == 0) f.seq = __ldcg(g.seq_in);
	return f;
}

// Entry t of the gradient step from its prefetched inputs.  T is read from
// L2: in the fused form other SMs wrote it in the same launch.
__device__ __forceinline__ void batch_gradient_from(const GradStepArgs &g, const double *T, int t, const GradPre &f)
{
	if (t < g.batch) g.out_ll[t] = f.inv_t ? -INFINITY : f.ll;
	if (t >= g.batch * g.nrefs) return;
	if (f.inv_b) {
		g.out_grad[t] = 0.0;
		return;
	}
	double Tp[NTAN];
#pragma unroll
	for (int k = 0; k < NTAN; k++) Tp[k] = __ldcg(T + (size_t)f.pi * NTAN + k);
	g.out_grad[t] = gradient_from_tangents(f.code, g.dev[f.pi].axrat, g.dev[f.pi], Tp);
}

__device__ __forceinline__ void batch_gradient_at(const GradStepArgs &g, const double *T, int t)
{
	batch_gradient_from(g, T, t, grad_prefetch(g, t));
}

// Called by one block per profile once that profile's T is written (or its
// blocks have nothing to reduce); the last of the gridDim.y calls runs the
// gradient step with all its threads.  Writers of T fence before the call.
// f: grad_prefetch(g, threadIdx.x), loaded by the caller.
__device__ __forceinline__ void jac_gradient_tail(const GradStepArgs &g, unsigned *ticket, const double *T,
                                                  const GradPre &f)
{
	__shared__ bool s_all;
	__syncthreads();
	if (threadIdx.x == 0) s_all = atomicAdd(ticket, 1u) == gridDim.y - 1;
	__syncthreads();
	if (!s_all) return;
	__threadfence();
	const int n = g.batch * max(g.nrefs, 1);
	if ((int)threadIdx.x < n) batch_gradient_from(g, T, threadIdx.x, f);
	for (int t = threadIdx.x + blockDim.x; t < n; t += blockDim.x) batch_gradient_at(g, T, t);
	if (g.ctrl_out) {
		if ((int)threadIdx.x < g.ctrl_words) g.ctrl_out[threadIdx.x] = f.ctrl;
		for (int i = threadIdx.x + blockDim.x; i < g.ctrl_words; i += blockDim.x) g.ctrl_out[i] = __ldcg(g.ctrl_in + i);
	}
	if (threadIdx.x == 0) *ticket = 0;
	if (g.seq_out) {
		// the results reach host memory before the word that announces them
		__threadfence_system();
		__syncthreads();
		if (threadIdx.x == 0) *reinterpret_cast<volatile unsigned *>(g.seq_out) = f.seq;
	}
}

// sum over pixels of g(pixel) * J_k(pixel) for each radial profile:
// blockIdx.y = profile, blockIdx.x strides over the pixel tiles of
// k_pixels32 (32 x 8, one pixel per thread), two tiles per step with every
// load issued before the products; tiles the profile does not reach
// (tile_culled, as the render decided them) are skipped, their planes never
// written.  About one wave of four blocks per SM (at most 64 registers with
// FP32 planes), so the last block to finish is not a second wave's.  Each
// block writes its NTAN sums to `partials`; the block that finishes last (an
// atomic ticket per profile, no waiting) adds the partials in block order and
// resets the ticket, so the result does not depend on block scheduling.
template <int NT, class JT>
__global__ void __launch_bounds__(256, (NT <= 9 && sizeof(JT) == 4) ? 4 : 2) k_jac_reduce(const JT *__restrict__ jac, const float *__restrict__ g_conv,
                                                    const float *__restrict__ g_plain,
                                                    const FProfile *__restrict__ profiles,
                                                    const int *__restrict__ prof_batch, unsigned width,
                                                    unsigned height, double sx, double sy, int nt,
                                                    double *__restrict__ partials, unsigned *__restrict__ tickets,
                                                    double *__restrict__ out, GradStepArgs grad,
                                                    unsigned *__restrict__ grad_ticket,
                                                    const int2 *__restrict__ extent)
{
	pdl_enter();
	constexpr int U = 2;
	const int pi = blockIdx.y;
	const FProfile &p = profiles[pi];
	if (!is_radial_kind(p.kind)) {
		if (grad_ticket && blockIdx.x == 0) jac_gradient_tail(grad, grad_ticket, out, grad_prefetch(grad, threadIdx.x));
		return;
	}
	const int nk = tangent_count(p.kind);  // <= nt <= NT
	const int b = prof_batch[pi];
	const size_t npix = (size_t)width * height;
	const float *g = (p.target == 0 ? g_conv : g_plain) + (size_t)b * npix;
	const JT *jp = jac + (size_t)pi * nt * npix;
	double acc[NT];
#pragma unroll
	for (int k = 0; k < NT; k++) acc[k] = 0.0;
	// U pixels per thread per step, every load issued before the products
	auto step = [&](const bool (&in)[U], const size_t (&pix)[U]) {
		float gv[U];
		JT jv[U][NT];
#pragma unroll
		for (int u = 0; u < U; u++) {
			gv[u] = in[u] ? g[pix[u]] : 0.f;
#pragma unroll
			for (int k = 0; k < NT; k++) jv[u][k] = (in[u] && k < nk) ? jp[(size_t)k * npix + pix[u]] : JT(0);
		}
#pragma unroll
		for (int u = 0; u < U; u++)
			if (gv[u] != 0.f) {
#pragma unroll
				for (int k = 0; k < NT; k++) {
					// FP64 planes carry sums an FP32 product would round away;
					// with FP32 planes the FP32 product is as exact as its factors
					if constexpr (sizeof(JT) == 8) acc[k] += (double)gv[u] * jv[u][k];
					else acc[k] += (double)(gv[u] * jv[u][k]);
				}
			}
	};
	// the planes end at the batch entry's extent (launch_pixels32)
	const unsigned ew = extent ? min(width, (unsigned)extent[b].x) : width;
	const unsigned eh = extent ? min(height, (unsigned)extent[b].y) : height;
	if (ew == width && eh == height && tiles_all_reached(p, width, height, sx, sy)) {
		// every tile holds planes: a plain stride over the pixels (no tile
		// padding at the right edge, no per-tile test)
		const unsigned stride = gridDim.x * blockDim.x * U;
		for (unsigned t0 = blockIdx.x * blockDim.x * U + threadIdx.x; t0 < npix; t0 += stride) {
			bool in[U];
			size_t pix[U];
#pragma unroll
			for (int u = 0; u < U; u++) {
				pix[u] = t0 + u * blockDim.x;
				in[u] = pix[u] < npix;
			}
			step(in, pix);
		}
	}
	else {
		// the block's tiles are blockIdx.x * U + j * gridDim.x * U + u (spread
		// over the drawing, so that the reached ones are shared out evenly);
		// each round, one thread per tile tests it and the reached ones are
		// listed in thread order, then the block walks the list U tiles a step
		__shared__ uint32_t s_tile[PIX_TILE_W * PIX_TILE_H];  // (ty << 16) | tx
		__shared__ int s_cnt[PIX_TILE_W * PIX_TILE_H / 32];
		const int tl = threadIdx.x & 31, tw = threadIdx.x >> 5;
		const unsigned tiles_x = (width + PIX_TILE_W - 1) / PIX_TILE_W;
		const unsigned ntiles = tiles_x * ((height + PIX_TILE_H - 1) / PIX_TILE_H);
		const unsigned lx = threadIdx.x % PIX_TILE_W, ly = threadIdx.x / PIX_TILE_W;
		const unsigned stride = gridDim.x * U, first = blockIdx.x * U;
		const unsigned count = first < ntiles ? ((ntiles - 1 - first) / stride + 1) * U : 0;
		for (unsigned c0 = 0; c0 < count; c0 += blockDim.x) {
			const unsigned c = c0 + threadIdx.x;
			bool keep = false;
			uint32_t code = 0;
			if (c < count) {
				const unsigned t = first + (c / U) * stride + (c % U);
				if (t < ntiles) {
					const unsigned ty = t / tiles_x, tx = t - ty * tiles_x;
					keep = tx * PIX_TILE_W < ew && ty * PIX_TILE_H < eh &&
					       !tile_culled(p, tx * PIX_TILE_W, ty * PIX_TILE_H, width, height, sx, sy);
					code = (ty << 16) | tx;
				}
			}
			const unsigned ballot = __ballot_sync(0xffffffffu, keep);
			if (tl == 0) s_cnt[tw] = __popc(ballot);
			__syncthreads();
			int before = 0, total = 0;
#pragma unroll
			for (int w = 0; w < PIX_TILE_W * PIX_TILE_H / 32; w++) {
				before += w < tw ? s_cnt[w] : 0;
				total += s_cnt[w];
			}
			if (keep) s_tile[before + __popc(ballot & ((1u << tl) - 1u))] = code;
			__syncthreads();
			for (int k = 0; k < total; k += U) {
				bool in[U];
				size_t pix[U];
#pragma unroll
				for (int u = 0; u < U; u++) {
					in[u] = k + u < total;
					pix[u] = 0;
					if (in[u]) {
						const uint32_t tc = s_tile[k + u];
						const unsigned i = (tc & 0xffffu) * PIX_TILE_W + lx, j = (tc >> 16) * PIX_TILE_H + ly;
						in[u] = i < ew && j < eh;
						pix[u] = (size_t)j * width + i;
					}
				}
				step(in, pix);
			}
			__syncthreads();  // the next round rewrites s_tile and s_cnt
		}
	}
	__shared__ double s_red[NT][8];
	__shared__ bool s_last;
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < NT; k++) {
		double v = warp_sum(acc[k]);
		if (lane == 0) s_red[k][wid] = v;
	}
	__syncthreads();
	double *mine = partials + ((size_t)pi * gridDim.x + blockIdx.x) * NTAN;
	if (threadIdx.x < NT) {
		double v = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += s_red[threadIdx.x][w];
		mine[threadIdx.x] = v;
		__threadfence();
	}
	__syncthreads();
	if (threadIdx.x == 0) s_last = atomicAdd(&tickets[pi], 1u) == gridDim.x - 1;
	__syncthreads();
	if (!s_last) return;
	__threadfence();
	// (the gradient step's own inputs travel with the partials)
	GradPre f;
	if (grad_ticket) f = grad_prefetch(grad, threadIdx.x);
	// the last block merges the partials with all its threads: thread t adds
	// blocks t, t + 256, ... in order, then warps and the block reduce in a
	// fixed order, so the result still does not depend on scheduling
	const volatile double *all = partials + (size_t)pi * gridDim.x * NTAN;
	double v[NT];
#pragma unroll
	for (int k = 0; k < NT; k++) v[k] = 0.0;
	for (unsigned blk = threadIdx.x; blk < gridDim.x; blk += blockDim.x)
#pragma unroll
		for (int k = 0; k < NT; k++)
			if (k < nk) v[k] += all[(size_t)blk * NTAN + k];
#pragma unroll
	for (int k = 0; k < NT; k++) {
		const double w = warp_sum(v[k]);
		if (lane == 0) s_red[k][wid] = w;
	}
	__syncthreads();
	if (threadIdx.x < NT) {
		double t = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += s_red[threadIdx.x][w];
		out[(size_t)pi * NTAN + threadIdx.x] = t;
		if (grad_ticket) __threadfence();
	}
	if (threadIdx.x == 0) tickets[pi] = 0;
	if (grad_ticket) jac_gradient_tail(grad, grad_ticket, out, f);
}

// Scatter the residual weights w (cropped grid) into the padded grid of the
// unconvolved image: g_plain(u) = w(u - pad).
__global__ void k_embed_seed(const float *__restrict__ w, unsigned ow, unsigned oh, unsigned padx, unsigned pady,
                             unsigned dw, unsigned dh, float *__restrict__ g_plain)
{
	pdl_enter();
	const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
	const unsigned j = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (i >= dw || j >= dh) return;
	float v = 0.f;
	if (i >= padx && j >= pady && i - padx < ow && j - pady < oh) v = w[(size_t)b * ow * oh + (i - padx) + (j - pady) * ow];
	g_plain[(size_t)b * dw * dh + i + j * dw] = v;
}

__global__ void k_crop32(const float *__restrict__ src, unsigned sw, unsigned ox, unsigned oy,
                         float *__restrict__ out, unsigned ow, unsigned oh, const float *__restrict__ add,
                         unsigned src_stride)
{
	pdl_enter();
	unsigned i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (i >= ow || j >= oh) return;
	size_t s = (size_t)b * src_stride + (i + ox) + (size_t)(j + oy) * sw;
	float v = src[s];
	if (add) v += add[s];
	out[(size_t)b * ow * oh + i + (size_t)j * ow] = v;
}

static inline unsigned cdiv(unsigned a, unsigned b) { return (a + b - 1) / b; }

// The start of one small FP32 evaluation in one launch: the staged profile
// scalars are read straight from pinned host memory (mapped into the device's
// address space) into their device buffer, and the queue's control words are
// zeroed.  This replaces a host-to-device copy and a memset, which cannot
// overlap the kernels around them the way a programmatic launch does.
__global__ void k_stage_in(uint4 *__restrict__ dst, const uint4 *__restrict__ src, size_t n16,
                           uint32_t *__restrict__ ctrl, int ctrl_words)
{
	pdl_enter();
	const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x, step = (size_t)gridDim.x * blockDim.x;
	for (size_t i = t; i < n16; i += step) dst[i] = src[i];
	for (size_t i = t; i < (size_t)ctrl_words; i += step) ctrl[i] = 0u;
}

cudaError_t launch_stage_in(void *dst, const void *host_src, size_t bytes, uint32_t *ctrl, int ctrl_words,
                            cudaStream_t s)
{
	const size_t n16 = bytes / 16;
	const unsigned blocks = (unsigned)std::min<size_t>(std::max<size_t>((n16 + 255) / 256, 1), 148);
	note_launches(1);
	return launch_pdl(k_stage_in, dim3(blocks), dim3(256), 0, s, static_cast<uint4 *>(dst),
	                  static_cast<const uint4 *>(host_src), n16, ctrl, ctrl_words);
}

cudaError_t launch_pixels32(const FProfile *profiles, const int *prof_begin, int batch, unsigned width,
                            unsigned height, double sx, double sy, float *img_conv, float *img_plain, JacPlanes jac,
                            int nt, bool all_kinds, const QueueSet &q, cudaStream_t s, const uint8_t *mask,
                            const int2 *extent)
{
	dim3 block(PIX_TILE_W, PIX_TILE_H), grid(cdiv(width, PIX_TILE_W), cdiv(height, PIX_TILE_H), batch);
	note_launches(1);
	if (jac.p && jac.fp64) {
		auto k = all_kinds ? k_pixels32<true, true, double> : k_pixels32<false, true, double>;
		return launch_pdl(k, grid, block, 0, s, profiles, prof_begin, width, height, sx, sy, img_conv, img_plain,
		                  static_cast<double *>(jac.p), nt, q, mask, extent);
	}
	if (!jac.p) {
		auto k = all_kinds ? k_pixels32_listed<true> : k_pixels32_listed<false>;
		dim3 lgrid(cdiv(width, 32), cdiv(height, 2 * LISTED_ROWS), batch);
		return launch_pdl(k, lgrid, dim3(32, LISTED_ROWS), 0, s, profiles, prof_begin, width, height, sx, sy, img_conv,
		                  img_plain, q, mask);
	}
	auto k = all_kinds ? k_pixels32<true, true, float> : k_pixels32<false, true, float>;
	return launch_pdl(k, grid, block, 0, s, profiles, prof_begin, width, height, sx, sy, img_conv, img_plain,
	                  static_cast<float *>(jac.p), nt, q, mask, extent);
}

// Kind grouping of one wide level's items (models with profiles of every
// kind): the level kernel then takes the items kind by kind, so the warps
// resident on an SM run one profile function at a time instead of all six
// (the code of all six does not fit the instruction cache).  Each block
// takes a contiguous range of items: it counts kinds in shared memory,
// reserves its slots per kind with one global atomic per kind (after the
// histogram pass fixed the kind bases), then scatters the item indices.
constexpr int KG_ITEMS_PER_BLOCK = 2048;

__global__ void k_kind_hist(const FProfile *__restrict__ profiles, QueueSet q, int level)
{
	pdl_enter();
	const uint32_t n = min(q.counts[level], q.cap[level]);
	const SubItem *items = q.items + q.off[level];
	__shared__ uint32_t s_h[N_RADIAL_KINDS];
	if (threadIdx.x < N_RADIAL_KINDS) s_h[threadIdx.x] = 0;
	__syncthreads();
	const uint32_t i0 = blockIdx.x * KG_ITEMS_PER_BLOCK, i1 = min(n, i0 + KG_ITEMS_PER_BLOCK);
	for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
		const int k = profiles[items[i].profile].kind - PK_SERSIC;
		if (k >= 0 && k < N_RADIAL_KINDS) atomicAdd(&s_h[k], 1u);
	}
	__syncthreads();
	uint32_t *hist = q.counts + KIND_CTR + level * 2 * N_RADIAL_KINDS;
	if (threadIdx.x < N_RADIAL_KINDS && s_h[threadIdx.x]) atomicAdd(&hist[threadIdx.x], s_h[threadIdx.x]);
}

__global__ void k_kind_scatter(const FProfile *__restrict__ profiles, QueueSet q, int level)
{
	pdl_enter();
	const uint32_t n = min(q.counts[level], q.cap[level]);
	const SubItem *items = q.items + q.off[level];
	const uint32_t *hist = q.counts + KIND_CTR + level * 2 * N_RADIAL_KINDS;
	uint32_t *cursor = q.counts + KIND_CTR + level * 2 * N_RADIAL_KINDS + N_RADIAL_KINDS;
	__shared__ uint32_t s_n[N_RADIAL_KINDS], s_at[N_RADIAL_KINDS];
	if (threadIdx.x < N_RADIAL_KINDS) s_n[threadIdx.x] = 0;
	__syncthreads();
	const uint32_t i0 = blockIdx.x * KG_ITEMS_PER_BLOCK, i1 = min(n, i0 + KG_ITEMS_PER_BLOCK);
	for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
		const int k = profiles[items[i].profile].kind - PK_SERSIC;
		if (k >= 0 && k < N_RADIAL_KINDS) atomicAdd(&s_n[k], 1u);
	}
	__syncthreads();
	if (threadIdx.x < N_RADIAL_KINDS) {
		uint32_t base = 0;
		for (int k = 0; k < (int)threadIdx.x; k++) base += hist[k];
		s_at[threadIdx.x] = s_n[threadIdx.x] ? base + atomicAdd(&cursor[threadIdx.x], s_n[threadIdx.x]) : 0;
	}
	__syncthreads();
	uint32_t *perm = q.perm + q.off[level];
	for (uint32_t i = i0 + threadIdx.x; i < i1; i += blockDim.x) {
		const int k = profiles[items[i].profile].kind - PK_SERSIC;
		// every queued item is a radial profile's; an out-of-range kind would
		// leave its slot to the identity
		const uint32_t pos = (k >= 0 && k < N_RADIAL_KINDS) ? atomicAdd(&s_at[k], 1u) : i;
		perm[pos] = i;
	}
}

template <class JT>
cudaError_t levels32(const FProfile *profiles, int n_levels, unsigned npix, float *img_conv, float *img_plain, JT *jac,
                     int nt, bool all_kinds, int cusps, const QueueSet &q, cudaStream_t s)
{
	const int wide = n_levels < 3 ? n_levels : 3;
	for (int l = 0; l < wide; l++) {
		if (q.perm) {
			// grid over the level's capacity (its count is only known on the device)
			const unsigned blocks = q.cap[l] / KG_ITEMS_PER_BLOCK + 1;
			cudaError_t e = launch_pdl(k_kind_hist, dim3(blocks), dim3(256), 0, s, profiles, q, l);
			if (e == cudaSuccess) e = launch_pdl(k_kind_scatter, dim3(blocks), dim3(256), 0, s, profiles, q, l);
			note_launches(2);
			if (e != cudaSuccess) return e;
		}
		auto k = all_kinds ? (jac ? k_level32<true, true, false, JT> : k_level32<true, false, false, JT>)
		                   : (jac ? k_level32<false, true, false, JT> : k_level32<false, false, false, JT>);
		cudaError_t e = launch_pdl(k, dim3(148 * 8), dim3(256), 0, s, profiles, l, npix, img_conv, img_plain, jac, nt, q);
		if (e != cudaSuccess) return e;
	}
	note_launches(wide);
	if (n_levels > wide && cusps > DEEP_ONE_CTA_MAX_CUSPS) {
		// many cusps (a large field, a batch): one grid-wide launch per level
		auto k = all_kinds ? (jac ? k_level32<true, true, true, JT> : k_level32<true, false, true, JT>)
		                   : (jac ? k_level32<false, true, true, JT> : k_level32<false, false, true, JT>);
		for (int l = wide; l < n_levels; l++) {
			cudaError_t e =
			    launch_pdl(k, dim3(148 * 8), dim3(256), 0, s, profiles, l, npix, img_conv, img_plain, jac, nt, q);
			if (e != cudaSuccess) return e;
		}
		note_launches(n_levels - wide);
	}
	else if (n_levels > wide) {
		auto k = all_kinds ? (jac ? k_deep_levels32<true, true, JT> : k_deep_levels32<true, false, JT>)
		                   : (jac ? k_deep_levels32<false, true, JT> : k_deep_levels32<false, false, JT>);
		cudaError_t e = launch_pdl(k, dim3(1), dim3(512), 0, s, profiles, wide, n_levels, npix, img_conv, img_plain, jac,
		                           nt, q);
		note_launches(1);
		if (e != cudaSuccess) return e;
	}
	return cudaGetLastError();
}

cudaError_t launch_levels32(const FProfile *profiles, int n_levels, unsigned npix, float *img_conv, float *img_plain,
                            JacPlanes jac, int nt, bool all_kinds, int cusps, const QueueSet &q, cudaStream_t s)
{
	if (jac.p && jac.fp64)
		return levels32<double>(profiles, n_levels, npix, img_conv, img_plain, static_cast<double *>(jac.p), nt,
		                        all_kinds, cusps, q, s);
	return levels32<float>(profiles, n_levels, npix, img_conv, img_plain, static_cast<float *>(jac.p), nt, all_kinds,
	                       cusps, q, s);
}

unsigned jac_reduce_blocks(unsigned width, unsigned height, int n_profiles)
{
	// about one wave of 4 blocks per SM in all, and the same number of
	// two-tile steps for every block (a block with one step more than the
	// others is the launch's tail)
	const unsigned tiles = cdiv(width, PIX_TILE_W) * cdiv(height, PIX_TILE_H);
	const unsigned target = cdiv(148u * 4u, (unsigned)n_profiles);
	const unsigned steps = std::max(1u, (unsigned)((double)tiles / (2.0 * target) + 0.5));
	return std::max(1u, cdiv(tiles, 2 * steps));
}

cudaError_t launch_jac_reduce(JacPlanes jac, const float *g_conv, const float *g_plain, const FProfile *profiles,
                              const int *prof_batch, int n_profiles, unsigned width, unsigned height, double sx,
                              double sy, int nt, double *partials, unsigned *tickets, double *out, cudaStream_t s,
                              const GradStepArgs *grad, const int2 *extent)
{
	const unsigned bx = jac_reduce_blocks(width, height, n_profiles);
	const GradStepArgs g = grad ? *grad : GradStepArgs{};
	unsigned *gt = grad ? tickets + n_profiles : (unsigned *)nullptr;
	note_launches(1);
	if (jac.fp64) {
		auto k = nt <= 9 ? k_jac_reduce<9, double> : k_jac_reduce<NTAN, double>;
		return launch_pdl(k, dim3(bx, n_profiles), dim3(PIX_TILE_W * PIX_TILE_H), 0, s,
		                  static_cast<const double *>(jac.p), g_conv, g_plain, profiles, prof_batch, width, height, sx,
		                  sy, nt, partials, tickets, out, g, gt, extent);
	}
	auto k = nt <= 9 ? k_jac_reduce<9, float> : k_jac_reduce<NTAN, float>;
	return launch_pdl(k, dim3(bx, n_profiles), dim3(PIX_TILE_W * PIX_TILE_H), 0, s, static_cast<const float *>(jac.p),
	                  g_conv, g_plain, profiles, prof_batch, width, height, sx, sy, nt, partials, tickets, out, g, gt,
	                  extent);
}

cudaError_t launch_embed_seed(const float *w, unsigned ow, unsigned oh, unsigned padx, unsigned pady, unsigned dw,
                              unsigned dh, int batch, float *g_plain, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(dw, 32), cdiv(dh, 8), batch);
	cudaError_t e = launch_pdl(k_embed_seed, grid, block, 0, s, w, ow, oh, padx, pady, dw, dh, g_plain);
	note_launches(1);
	if (e != cudaSuccess) return e;
	return cudaGetLastError();
}

// libprofit's psf profile (psf.cpp:58-145) in the FP32 pipeline: the FP64
// area-overlap stamp of the normalised PSF image that k_psf_stamp64 draws
// (same ranges and quirks), and for the adjoint its derivatives in the
// centre.  The stamp origin moves with xcen (px) and ycen (py), so for each
// overlap ix = min(x + sx, psf_x + psf_sx) - max(x, psf_x),
// d ix / d px = [psf_x + psf_sx < x + sx] - [psf_x > x] (likewise in y);
// PSF pixels entering or leaving a range do so at zero overlap.
struct PsfStamp {
	double origin_x, origin_y;
	unsigned x0, y0, nx, ny;
};

__device__ __forceinline__ bool psf_stamp_geom(const DevProfile &d, unsigned psf_w, unsigned psf_h, double psf_sx,
                                               double psf_sy, double scale_x, double scale_y, double offx, double offy,
                                               unsigned width, unsigned height, PsfStamp &g)
{
	g.origin_x = d.px + offx * scale_x - psf_w * psf_sx / 2;
	const double end_x = d.px + offy * scale_y + psf_w * psf_sx / 2;
	g.origin_y = d.py + offx * scale_x - psf_h * psf_sy / 2;
	const double end_y = d.py + offy * scale_y + psf_h * psf_sy / 2;
	g.x0 = bind_u(g.origin_x / scale_x, width - 1);
	g.y0 = bind_u(g.origin_y / scale_y, height - 1);
	const unsigned x1 = bind_u(end_x / scale_x, width - 1), y1 = bind_u(end_y / scale_y, height - 1);
	if (x1 < g.x0 || y1 < g.y0) return false;
	g.nx = x1 - g.x0 + 1;
	g.ny = y1 - g.y0 + 1;
	return true;
}

// Stamp value at target pixel (pix_x, pix_y) (flux 1); with D also its
// derivatives in px and py.
template <bool D>
__device__ __forceinline__ double psf_stamp_pixel(const double *__restrict__ psf, unsigned psf_w, unsigned psf_h,
                                                  double psf_sx, double psf_sy, double scale_x, double scale_y,
                                                  const PsfStamp &g, unsigned pix_x, unsigned pix_y, double &dvx,
                                                  double &dvy)
{
	const double y = pix_y * scale_y, x = pix_x * scale_x;
	const int px0 = (int)bind_u(floor((x - g.origin_x) / psf_sx), psf_w - 1);
	int px1 = (int)bind_u(floor((x - g.origin_x + scale_x) / psf_sx), psf_h - 1);
	int py0 = (int)bind_u(floor((y - g.origin_y) / psf_sy), psf_w - 1);
	const int py1 = (int)bind_u(floor((y - g.origin_y + scale_y) / psf_sy), psf_h - 1);
	px1 = min(px1, (int)psf_w - 1);
	py0 = min(py0, (int)psf_h - 1);
	double val = 0;
	dvx = dvy = 0;
	for (int yy = py0; yy <= py1; yy++) {
		const double psf_y = yy * psf_sy + g.origin_y;
		const double iy = fmin(y + scale_y, psf_y + psf_sy) - fmax(y, psf_y);
		const double diy = (psf_y + psf_sy < y + scale_y ? 1.0 : 0.0) - (psf_y > y ? 1.0 : 0.0);
		for (int xx = px0; xx <= px1; xx++) {
			const double psf_x = xx * psf_sx + g.origin_x;
			const double ix = fmin(x + scale_x, psf_x + psf_sx) - fmax(x, psf_x);
			const double w = psf[xx + yy * psf_w] / (psf_sx * psf_sy);
			val += psf[xx + yy * psf_w] * (ix * iy) / (psf_sx * psf_sy);
			if constexpr (D) {
				const double dix = (psf_x + psf_sx < x + scale_x ? 1.0 : 0.0) - (psf_x > x ? 1.0 : 0.0);
				dvx += w * dix * iy;
				dvy += w * ix * diy;
			}
		}
	}
	return val;
}

// Forward: every psf profile of batch entry blockIdx.y adds flux x stamp to
// its target image (after the radial pixel and level kernels).
__global__ void k_psf_stamp32(const DevProfile *__restrict__ dev, const int *__restrict__ prof_begin,
                              const double *__restrict__ psf, unsigned psf_w, unsigned psf_h, double psf_sx,
                              double psf_sy, double scale_x, double scale_y, double offx, double offy, unsigned width,
                              unsigned height, float *__restrict__ img_conv, float *__restrict__ img_plain)
{
	pdl_enter();
	const int b = blockIdx.y;
	const size_t npix = (size_t)width * height;
	for (int pi = prof_begin[b]; pi < prof_begin[b + 1]; pi++) {
		const DevProfile &d = dev[pi];
		if (d.kind != PK_PSF) continue;
		PsfStamp g;
		if (!psf_stamp_geom(d, psf_w, psf_h, psf_sx, psf_sy, scale_x, scale_y, offx, offy, width, height, g)) continue;
		float *img = (d.target == 0 ? img_conv : img_plain) + (size_t)b * npix;
		for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < g.nx * g.ny; t += gridDim.x * blockDim.x) {
			const unsigned pix_x = g.x0 + t % g.nx, pix_y = g.y0 + t / g.nx;
			double dvx, dvy;
			const double val = psf_stamp_pixel<false>(psf, psf_w, psf_h, psf_sx, psf_sy, scale_x, scale_y, g, pix_x,
			                                          pix_y, dvx, dvy);
			atomicAdd(&img[pix_x + (size_t)pix_y * width], (float)(val * d.psf_flux));
		}
	}
}

// Adjoint: block (blockIdx.x, blockIdx.y) = local profile index and batch
// entry; a psf profile's T[0..2] = sum over its stamp of g x (stamp,
// d stamp / d xcen, d stamp / d ycen), summed in FP64 in a fixed order.
__global__ void __launch_bounds__(256)
    k_psf_adjoint32(const DevProfile *__restrict__ dev, const int *__restrict__ prof_begin,
                    const double *__restrict__ psf, unsigned psf_w, unsigned psf_h, double psf_sx, double psf_sy,
                    double scale_x, double scale_y, double offx, double offy, unsigned width, unsigned height,
                    const float *__restrict__ g_conv, const float *__restrict__ g_plain, double *__restrict__ T)
{
	pdl_enter();
	const int b = blockIdx.y, pi = prof_begin[b] + (int)blockIdx.x;
	if (pi >= prof_begin[b + 1]) return;
	const DevProfile &d = dev[pi];
	if (d.kind != PK_PSF) return;
	PsfStamp g;
	double acc[3] = {0, 0, 0};
	if (psf_stamp_geom(d, psf_w, psf_h, psf_sx, psf_sy, scale_x, scale_y, offx, offy, width, height, g)) {
		const float *gi = (d.target == 0 ? g_conv : g_plain) + (size_t)b * width * height;
		for (unsigned t = threadIdx.x; t < g.nx * g.ny; t += blockDim.x) {
			const unsigned pix_x = g.x0 + t % g.nx, pix_y = g.y0 + t / g.nx;
			const double gv = gi[pix_x + (size_t)pix_y * width];
			if (gv == 0.0) continue;
			double dvx, dvy;
			const double val = psf_stamp_pixel<true>(psf, psf_w, psf_h, psf_sx, psf_sy, scale_x, scale_y, g, pix_x,
			                                         pix_y, dvx, dvy);
			acc[0] += gv * val;
			acc[1] += gv * dvx;
			acc[2] += gv * dvy;
		}
	}
	__shared__ double s_red[3][8];
	const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < 3; k++) {
		const double v = warp_sum(acc[k]);
		if (lane == 0) s_red[k][wid] = v;
	}
	__syncthreads();
	if (threadIdx.x < 3) {
		double v = 0;
		for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += s_red[threadIdx.x][w];
		T[(size_t)pi * NTAN + threadIdx.x] = v;
	}
}

cudaError_t launch_psf_stamp32(const DevProfile *dev, const int *prof_begin, int batch, const double *psf,
                               unsigned psf_w, unsigned psf_h, double psf_sx, double psf_sy, double scale_x,
                               double scale_y, double offx, double offy, unsigned width, unsigned height,
                               float *img_conv, float *img_plain, cudaStream_t s)
{
	note_launches(1);
	return launch_pdl(k_psf_stamp32, dim3(16, batch), dim3(256), 0, s, dev, prof_begin, psf, psf_w, psf_h, psf_sx,
	                  psf_sy, scale_x, scale_y, offx, offy, width, height, img_conv, img_plain);
}

cudaError_t launch_psf_adjoint32(const DevProfile *dev, const int *prof_begin, int batch, int nprof_max,
                                 const double *psf, unsigned psf_w, unsigned psf_h, double psf_sx, double psf_sy,
                                 double scale_x, double scale_y, double offx, double offy, unsigned width,
                                 unsigned height, const float *g_conv, const float *g_plain, double *T, cudaStream_t s)
{
	note_launches(1);
	return launch_pdl(k_psf_adjoint32, dim3(nprof_max, batch), dim3(256), 0, s, dev, prof_begin, psf, psf_w, psf_h,
	                  psf_sx, psf_sy, scale_x, scale_y, offx, offy, width, height, g_conv, g_plain, T);
}

// The FP32 pipeline's model image from the convolved fine image, for the
// cases beyond one plain crop (Model::evaluate, model.cpp:307-334):
//   fine(i, j) = plain drawing pixel where the drawing mask is 0 and the
//                convolution was masked (sel, drawing size, optional);
//   out(I, J)  = sum of the fs x fs fine pixels of the output pixel (the
//                finesampled image summed down), 0 where the output mask
//                (mask_out, output size, optional) is 0.
// Strides: fine nfine, plain npix, out nout per batch entry (blockIdx.z).
__global__ void k_model_finish32(const double *__restrict__ fine, unsigned cw, unsigned ch, size_t nfine,
                                 const float *__restrict__ plain, const uint8_t *__restrict__ sel, unsigned dw,
                                 size_t npix, unsigned padx, unsigned pady, unsigned fs,
                                 const uint8_t *__restrict__ mask_out, double *__restrict__ out, unsigned ow,
                                 unsigned oh, size_t nout)
{
	pdl_enter();
	const unsigned I = blockIdx.x * blockDim.x + threadIdx.x, J = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (I >= ow || J >= oh) return;
	fine += (size_t)b * nfine;
	plain += (size_t)b * npix;
	double v = 0;
	for (unsigned row = J * fs; row < min((J + 1) * fs, ch); row++)
		for (unsigned col = I * fs; col < min((I + 1) * fs, cw); col++) {
			const size_t d = (col + padx) + (size_t)(row + pady) * dw;
			v += (sel && !sel[d]) ? (double)plain[d] : fine[col + (size_t)row * cw];
		}
	if (mask_out && !mask_out[I + (size_t)J * ow]) v = 0.0;
	out[(size_t)b * nout + I + (size_t)J * ow] = v;
}

// Adjoint of k_model_finish32 and of the crop: from dlogL/dout (w, output
// size) to the seed of the convolved image on the fine crop window (seed_conv,
// cw x ch) and to dlogL/d(unconvolved drawing pixel) (g_plain, drawing size,
// 0 outside the crop window).  A fine pixel receives its output pixel's w
// (the sum down), 0 where the output mask is 0; its convolved part also 0
// where the masked convolution kept the plain pixel.
__global__ void k_seed_finish32(const float *__restrict__ w, unsigned ow, unsigned oh, size_t nout,
                                const uint8_t *__restrict__ mask_out, const uint8_t *__restrict__ sel, unsigned fs,
                                unsigned cw, unsigned ch, size_t nfine, unsigned padx, unsigned pady, unsigned dw,
                                unsigned dh, size_t npix, float *__restrict__ seed_conv, float *__restrict__ g_plain)
{
	pdl_enter();
	const unsigned u = blockIdx.x * blockDim.x + threadIdx.x, v = blockIdx.y * blockDim.y + threadIdx.y;
	const int b = blockIdx.z;
	if (u >= dw || v >= dh) return;
	const size_t d = u + (size_t)v * dw;
	float g = 0.f;
	if (u >= padx && v >= pady && u - padx < cw && v - pady < ch) {
		const unsigned i = u - padx, j = v - pady;
		const size_t o = i / fs + (size_t)(j / fs) * ow;
		g = (mask_out && !mask_out[o]) ? 0.f : w[(size_t)b * nout + o];
		seed_conv[(size_t)b * nfine + i + (size_t)j * cw] = (sel && !sel[d]) ? 0.f : g;
	}
	g_plain[(size_t)b * npix + d] = g;
}

cudaError_t launch_model_finish32(const double *fine, unsigned cw, unsigned ch, const float *plain, const uint8_t *sel,
                                  unsigned dw, unsigned dh, unsigned padx, unsigned pady, unsigned fs,
                                  const uint8_t *mask_out, double *out, unsigned ow, unsigned oh, int batch,
                                  cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(ow, 32), cdiv(oh, 8), batch);
	note_launches(1);
	return launch_pdl(k_model_finish32, grid, block, 0, s, fine, cw, ch, (size_t)cw * ch, plain, sel, dw,
	                  (size_t)dw * dh, padx, pady, fs, mask_out, out, ow, oh, (size_t)ow * oh);
}

cudaError_t launch_seed_finish32(const float *w, unsigned ow, unsigned oh, const uint8_t *mask_out, const uint8_t *sel,
                                 unsigned fs, unsigned cw, unsigned ch, unsigned padx, unsigned pady, unsigned dw,
                                 unsigned dh, int batch, float *seed_conv, float *g_plain, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(dw, 32), cdiv(dh, 8), batch);
	note_launches(1);
	return launch_pdl(k_seed_finish32, grid, block, 0, s, w, ow, oh, (size_t)ow * oh, mask_out, sel, fs, cw, ch,
	                  (size_t)cw * ch, padx, pady, dw, dh, (size_t)dw * dh, seed_conv, g_plain);
}

// FP32 taps, FP64 column accumulation; FP32 output (adjoint) or FP64 output
// (forward model, so the likelihood sees the full-precision sum).
template <class TOut>
static cudaError_t conv32_any(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                              TOut *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                              int batch, int batch_src_stride, int batch_out_stride, double *scratch,
                              size_t scratch_bytes, int batch_k_stride, cudaStream_t s)
{
	note_launches(1);
	static const ConvCandidate cands[] = {
	    // packed-FMA kernels: (lanes per row, rows per thread, row groups, column groups, column splits)
	    {Conv3Variant<TOut, 32, 8, 2, 4, 1>::smem, Conv3Variant<TOut, 32, 8, 2, 4, 1>::run},
	    {Conv3Variant<TOut, 32, 8, 4, 1, 1>::smem, Conv3Variant<TOut, 32, 8, 4, 1, 1>::run},
	    {Conv3Variant<TOut, 32, 12, 4, 1, 1>::smem, Conv3Variant<TOut, 32, 12, 4, 1, 1>::run},
	    {Conv3Variant<TOut, 32, 8, 1, 8, 1>::smem, Conv3Variant<TOut, 32, 8, 1, 8, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 2, 1, 1>::smem, Conv3Variant<TOut, 16, 8, 2, 1, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 4, 1, 1>::smem, Conv3Variant<TOut, 16, 8, 4, 1, 1>::run},
	    {Conv3Variant<TOut, 16, 12, 2, 1, 1>::smem, Conv3Variant<TOut, 16, 12, 2, 1, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 4, 1>::smem, Conv3Variant<TOut, 16, 8, 1, 4, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 8, 1>::smem, Conv3Variant<TOut, 16, 8, 1, 8, 1>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 4, 2>::smem, Conv3Variant<TOut, 16, 8, 1, 4, 2>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 4, 4>::smem, Conv3Variant<TOut, 16, 8, 1, 4, 4>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 2, 4>::smem, Conv3Variant<TOut, 16, 8, 1, 2, 4>::run},
	    {Conv3Variant<TOut, 16, 8, 2, 2, 2>::smem, Conv3Variant<TOut, 16, 8, 2, 2, 2>::run},
	    {Conv3Variant<TOut, 32, 8, 1, 4, 2>::smem, Conv3Variant<TOut, 32, 8, 1, 4, 2>::run},
	    // taller tiles: fewer CTAs, so that one image's grid fits the resident
	    // slots in one wave instead of leaving a partial second wave
	    {Conv3Variant<TOut, 32, 10, 1, 8, 1>::smem, Conv3Variant<TOut, 32, 10, 1, 8, 1>::run},
	    {Conv3Variant<TOut, 32, 12, 1, 8, 1>::smem, Conv3Variant<TOut, 32, 12, 1, 8, 1>::run},
	    {Conv3Variant<TOut, 32, 6, 1, 8, 1>::smem, Conv3Variant<TOut, 32, 6, 1, 8, 1>::run},
	    {Conv3Variant<TOut, 16, 10, 1, 8, 1>::smem, Conv3Variant<TOut, 16, 10, 1, 8, 1>::run},
	    // one-column-per-lane kernels
	    {ConvVariant<float, double, TOut, 8, 1, 8>::smem, ConvVariant<float, double, TOut, 8, 1, 8>::run},
	    {ConvVariant<float, double, TOut, 8, 2, 4>::smem, ConvVariant<float, double, TOut, 8, 2, 4>::run},
	    // fixed kernel heights (the 51x51 and 31x31 PSFs of the benchmark
	    // workloads): every tap of a column unrolled, no loop or tail
	    {Conv3Variant<TOut, 32, 10, 1, 8, 1, 51>::smem, Conv3Variant<TOut, 32, 10, 1, 8, 1, 51>::run},
	    {Conv3Variant<TOut, 16, 10, 1, 8, 1, 51>::smem, Conv3Variant<TOut, 16, 10, 1, 8, 1, 51>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 4, 1, 51>::smem, Conv3Variant<TOut, 16, 8, 1, 4, 1, 51>::run},
	    {Conv3Variant<TOut, 16, 8, 1, 8, 1, 51>::smem, Conv3Variant<TOut, 16, 8, 1, 8, 1, 51>::run},
	    {Conv3Variant<TOut, 32, 8, 4, 1, 1, 31>::smem, Conv3Variant<TOut, 32, 8, 4, 1, 1, 31>::run},
	    {Conv3Variant<TOut, 32, 12, 4, 1, 1, 31>::smem, Conv3Variant<TOut, 32, 12, 4, 1, 1, 31>::run},
	    // more rows per thread (fewer window loads per packed FMA), and
	    // 128-thread CTAs (five resident per SM instead of two)
	    {Conv3Variant<TOut, 32, 12, 1, 8, 1, 51>::smem, Conv3Variant<TOut, 32, 12, 1, 8, 1, 51>::run},
	    {Conv3Variant<TOut, 16, 12, 1, 8, 1, 51>::smem, Conv3Variant<TOut, 16, 12, 1, 8, 1, 51>::run},
	    {Conv3Variant<TOut, 32, 10, 1, 4, 1, 51>::smem, Conv3Variant<TOut, 32, 10, 1, 4, 1, 51>::run},
	    {Conv3Variant<TOut, 32, 8, 1, 8, 1, 51>::smem, Conv3Variant<TOut, 32, 8, 1, 8, 1, 51>::run},
	    // tensor-core kernels (tcgen05, 3xTF32): 32 output columns per tile,
	    // kernel rows split over 1, 2 or 4 CTAs.  Never picked by the
	    // autotuner, only when forced: on a 400x400 image with a 51x51 PSF they
	    // take 76-133 us against 35 us for the FMA kernels, and the tensor
	    // cores' FP32 accumulation leaves logL ~2e-7 and single gradient
	    // components up to ~9e-5 from the FP64 form (FMA kernels: 2e-8, 9e-6)
	    {ConvTcVariant<TOut, 32, 1>::smem, ConvTcVariant<TOut, 32, 1>::run, false},
	    {ConvTcVariant<TOut, 32, 2>::smem, ConvTcVariant<TOut, 32, 2>::run, false},
	    {ConvTcVariant<TOut, 32, 4>::smem, ConvTcVariant<TOut, 32, 4>::run, false},
	};
	ConvArgs a{src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, batch,
	           batch_src_stride, batch_out_stride, scratch, scratch_bytes, batch_k_stride};
	return conv_autotuned(cands, (int)(sizeof(cands) / sizeof(cands[0])), sizeof(TOut) == 8 ? 2 : 1, a, s);
}

size_t conv32_scratch_bytes(int ow, int oh, int batch)
{
	const size_t bytes = (size_t)ow * oh * batch * 4 * sizeof(double);  // up to 4 column splits
	return bytes <= ((size_t)64 << 20) ? bytes : 0;
}

cudaError_t launch_conv32(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                          float *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                          int batch, int batch_src_stride, int batch_out_stride, double *scratch, size_t scratch_bytes,
                          int batch_k_stride, cudaStream_t s)
{
	return conv32_any<float>(src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, batch,
	                         batch_src_stride, batch_out_stride, scratch, scratch_bytes, batch_k_stride, s);
}

cudaError_t launch_conv32_to64(const float *src, int sw, int sh, int ox, int oy, const float *K, int kw, int kh,
                               double *out, int ow, int oh, const float *add, int add_stride, int add_ox, int add_oy,
                               int batch, int batch_src_stride, int batch_out_stride, double *scratch,
                               size_t scratch_bytes, int batch_k_stride, cudaStream_t s)
{
	return conv32_any<double>(src, sw, sh, ox, oy, K, kw, kh, out, ow, oh, add, add_stride, add_ox, add_oy, batch,
	                          batch_src_stride, batch_out_stride, scratch, scratch_bytes, batch_k_stride, s);
}

cudaError_t launch_loglike32(const float *model, const double *data, const double *sigma, const uint8_t *region,
                             int n, int batch, int data_batch_stride, double2 *partials, int nparts, double *out,
                             float *wseed, cudaStream_t s)
{
	cudaError_t e = launch_pdl(k_loglike_partial<float>, dim3(nparts, batch), dim3(256), 0, s, model, data, sigma,
	                           region, n, partials, wseed, data_batch_stride);
	if (e == cudaSuccess) e = launch_pdl(k_loglike_final, dim3(batch), dim3(256), 0, s, partials, nparts, out);
	note_launches(2);
	return e;
}

cudaError_t launch_crop32(const float *src, unsigned sw, unsigned ox, unsigned oy, float *out, unsigned ow,
                          unsigned oh, const float *add, int batch, unsigned src_stride, cudaStream_t s)
{
	dim3 block(32, 8), grid(cdiv(ow, 32), cdiv(oh, 8), batch);
	note_launches(1);
	return launch_pdl(k_crop32, grid, block, 0, s, src, sw, ox, oy, out, ow, oh, add, src_stride);
}

// ---------------------------------------------------------------------------
// Batched proposals: device-side prologue and gradient assembly
// ---------------------------------------------------------------------------

// One thread per (proposal, profile): the model's parameters with this
// proposal's values written in, checked like RadialProfile::validate, then the
// FP64 scalar prologue (b_n, luminosity, Ie, auto-adjusted subsampling).  A
// proposal with an invalid profile is flagged and its profiles become null
// profiles, so nothing is drawn for it.
// Profile p of proposal b: the template with the proposal's values.
__device__ __forceinline__ ProfileParams proposal_params(const ProfileParams *__restrict__ tmpl, int p, int b,
                                                        const int *__restrict__ ref_profile,
                                                        const int *__restrict__ ref_offset, int nrefs,
                                                        const double *__restrict__ values)
{
	ProfileParams pp = tmpl[p];
	for (int r = 0; r < nrefs; r++)
		if (ref_profile[r] == p)
			*reinterpret_cast<double *>(reinterpret_cast<char *>(&pp) + ref_offset[r]) = values[(size_t)b * nrefs + r];
	return pp;
}

__global__ void k_batch_prologue(const ProfileParams *__restrict__ tmpl, int nprof, int batch,
                                 const int *__restrict__ ref_profile, const int *__restrict__ ref_offset, int nrefs,
                                 const double *__restrict__ values, ModelGeom g, DevProfile *__restrict__ dev,
                                 FProfile *__restrict__ fprof, int *__restrict__ invalid)
{
	pdl_enter();
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= batch * nprof) return;
	const int b = t / nprof, p = t - b * nprof;
	ProfileParams pp = proposal_params(tmpl, p, b, ref_profile, ref_offset, nrefs, values);
	if (!params_valid(pp)) {
		invalid[b] = 1;
		pp.kind = PK_NULL;
	}
	DevProfile d;
	derive_profile(pp, g, d);
	dev[t] = d;
	fprof[t] = to_fprofile(d, pp);
}

// One thread per (proposal, parameter): d logL / d parameter from the tangent
// reductions; invalid proposals get logL = -inf and a zero gradient.
__global__ void k_batch_gradient(const DevProfile *__restrict__ dev, int nprof, int batch,
                                 const int *__restrict__ ref_profile, const int *__restrict__ ref_code, int nrefs,
                                 const double *__restrict__ T, const double *__restrict__ ll, const int *__restrict__ invalid,
                                 double *__restrict__ out_ll, double *__restrict__ out_grad)
{
	pdl_enter();
	const GradStepArgs g = {dev, nprof, batch, nrefs, ref_profile, ref_code, ll, invalid, out_ll, out_grad,
	                        nullptr, nullptr, 0};
	batch_gradient_at(g, T, (int)(blockIdx.x * blockDim.x + threadIdx.x));
}

cudaError_t launch_batch_prologue(const ProfileParams *tmpl, int nprof, int batch, const int *ref_profile,
                                  const int *ref_offset, int nrefs, const double *values, const ModelGeom &g,
                                  DevProfile *dev, FProfile *fprof, int *invalid, cudaStream_t s)
{
	int n = batch * nprof;
	note_launches(1);
	return launch_pdl(k_batch_prologue, dim3((n + 127) / 128), dim3(128), 0, s, tmpl, nprof, batch, ref_profile,
	                  ref_offset, nrefs, values, g, dev, fprof, invalid);
}

cudaError_t launch_batch_gradient(const DevProfile *dev, int nprof, int batch, const int *ref_profile,
                                  const int *ref_code, int nrefs, const double *T, const double *ll,
                                  const int *invalid, double *out_ll, double *out_grad, cudaStream_t s)
{
	int n = batch * (nrefs > 1 ? nrefs : 1);
	note_launches(1);
	return launch_pdl(k_batch_gradient, dim3((n + 255) / 256), dim3(256), 0, s, dev, nprof, batch, ref_profile,
	                  ref_code, nrefs, T, ll, invalid, out_ll, out_grad);
}

// Catalogue batches: every galaxy brings its own profiles, so the prologue
// reads one parameter record per profile (validated when the galaxy was
// added) instead of a template plus a value matrix.
// pad[t]: the PSF padding of the bucket that draws profile t.
// The luminosity evaluations of the catalogue's core-Sersic, King, broken
// exponential and Ferrer profiles (lum_slot: the profile's own and +-h in each
// shape parameter), one thread per evaluation: each is a serial QUADPACK run,
// and one thread per profile ran up to eleven of them back to back.  A
// profile's slots sit in consecutive lanes, so a warp integrates one kind.
__global__ void k_cat_lum(const ProfileParams *__restrict__ params, int n, double *__restrict__ lum)
{
	pdl_enter();
	const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= (long long)n * LUM_SLOTS) return;
	const int pi = (int)(t / LUM_SLOTS), slot = (int)(t - (long long)pi * LUM_SLOTS);
	const ProfileParams pp = params[pi];
	if (slot < lum_slots(pp.kind)) lum[t] = lum_slot(pp, slot);
}

__global__ void k_cat_prologue(const ProfileParams *__restrict__ params, const int2 *__restrict__ pad, int n,
                               ModelGeom g, const double *__restrict__ lum, DevProfile *__restrict__ dev,
                               FProfile *__restrict__ fprof)
{
	pdl_enter();
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const ProfileParams pp = params[t];
	g.offx = pad[t].x;
	g.offy = pad[t].y;
	DevProfile d;
	derive_profile(pp, g, d, lum ? lum + (size_t)t * LUM_SLOTS : nullptr);
	dev[t] = d;
	fprof[t] = to_fprofile(d, pp);
}

// One thread per profile: d logL / d(every parameter of the profile) from its
// tangent reductions, in the order xcen, ycen, mag, ang, axrat, box, then the
// kind's shape parameters, written at grad_off[profile].
__global__ void k_cat_gradient(const DevProfile *__restrict__ dev, int n, const double *__restrict__ T,
                               const int *__restrict__ grad_off, double *__restrict__ grad)
{
	pdl_enter();
	const int t = blockIdx.x * blockDim.x + threadIdx.x;
	if (t >= n) return;
	const DevProfile &d = dev[t];
	if (!is_radial_kind(d.kind)) return;
	const double *Tp = T + (size_t)t * NTAN;
	double *out = grad + grad_off[t];
	const int codes[6] = {G_XCEN, G_YCEN, G_MAG, G_ANG, G_AXRAT, G_BOX};
	for (int c = 0; c < 6; c++) out[c] = gradient_from_tangents(codes[c], d.axrat, d, Tp);
	for (int k = 0; k < shape_count(d.kind); k++) out[6 + k] = gradient_from_tangents(G_SHAPE + k, d.axrat, d, Tp);
}

cudaError_t launch_cat_prologue(const ProfileParams *params, const int2 *pad, int n, const ModelGeom &g,
                                double *lum, DevProfile *dev, FProfile *fprof, cudaStream_t s)
{
	cudaError_t e = cudaSuccess;
	if (lum) {
		const long long nt = (long long)n * LUM_SLOTS;
		e = launch_pdl(k_cat_lum, dim3((unsigned)((nt + 127) / 128)), dim3(128), 0, s, params, n, lum);
		note_launches(1);
		if (e != cudaSuccess) return e;
	}
	note_launches(1);
	return launch_pdl(k_cat_prologue, dim3((n + 63) / 64), dim3(64), 0, s, params, pad, n, g, (const double *)lum, dev,
	                  fprof);
}

cudaError_t launch_cat_gradient(const DevProfile *dev, int n, const double *T, const int *grad_off, double *grad,
                                cudaStream_t s)
{
	note_launches(1);
	return launch_pdl(k_cat_gradient, dim3((n + 127) / 128), dim3(128), 0, s, dev, n, T, grad_off, grad);
}

__global__ void k_cat_scatter(const CatPiece *__restrict__ pieces, const double *__restrict__ stage,
                              double *__restrict__ data, double *__restrict__ sigma, uint8_t *__restrict__ region)
{
	const CatPiece pc = pieces[blockIdx.y];
	const long long n = (long long)pc.w * pc.rows;
	const double *d = stage + pc.src, *sg = d + n;
	for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
		const long long y = i / pc.w, x = i - y * pc.w;
		const unsigned long long o = pc.dst + (unsigned long long)y * pc.W + x;
		data[o] = d[i];
		sigma[o] = sg[i];
		region[o] = 1;
	}
}

cudaError_t launch_cat_scatter(const CatPiece *pieces, int n_pieces, int max_pixels, const double *stage,
                               double *data, double *sigma, uint8_t *region, cudaStream_t s)
{
	if (n_pieces <= 0) return cudaSuccess;
	if (n_pieces > 65535) return cudaErrorInvalidValue;
	note_launches(1);
	const unsigned gx = (unsigned)std::min(64, std::max(1, (max_pixels + 1023) / 1024));
	k_cat_scatter<<<dim3(gx, (unsigned)n_pieces), dim3(256), 0, s>>>(pieces, stage, data, sigma, region);
	return cudaGetLastError();
}

cudaError_t launch_loglike64_batch(const double *model, const double *data, const double *sigma,
                                   const uint8_t *region, int n, int batch, int data_batch_stride, double2 *partials,
                                   int nparts, double *out, float *wseed, cudaStream_t s, unsigned *tickets)
{
	if (tickets) {
		note_launches(1);
		return launch_pdl(k_loglike_fused<double>, dim3(nparts, batch), dim3(256), 0, s, model, data, sigma, region, n,
		                  partials, wseed, data_batch_stride, tickets, out);
	}
	cudaError_t e = launch_pdl(k_loglike_partial<double>, dim3(nparts, batch), dim3(256), 0, s, model, data, sigma,
	                           region, n, partials, wseed, data_batch_stride);
	if (e == cudaSuccess) e = launch_pdl(k_loglike_final, dim3(batch), dim3(256), 0, s, partials, nparts, out);
	note_launches(2);
	return e;
}

}  // namespace pf
