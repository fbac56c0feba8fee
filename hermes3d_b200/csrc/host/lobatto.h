// 1D hierarchical Lobatto shape functions and Gauss-Legendre rules (host).
//
// Lobatto functions follow the definitions used by the reference
// (src/shapeset/lobatto.h:80-109, src/shapeset/lobatto.cc:23-99):
//   L0(x) = (1 - x)/2,  L1(x) = (1 + x)/2,
//   L_k(x) = (P_k(x) - P_{k-2}(x)) / sqrt(2(2k-1))      for k >= 2,
//   L_k'(x) = sqrt((2k-1)/2) P_{k-1}(x),
// with P_n the Legendre polynomials (three-term recurrence).  The reference
// writes the same polynomials as (1-x^2)/4 times kernel functions phi_{k-2};
// the values agree to rounding.
//
// Gauss-Legendre rules are computed here to full double precision (Newton
// iteration on P_n in long double, mirrored so the rule is exactly
// symmetric).  The reference stores 14-digit tables (src/quadstd.cc:30-158);
// the two differ by ~1e-14 relative, well inside the parity tolerance.
// Point order is ascending, as in the reference tables; the 3D rule is the
// tensor product with x outermost and z innermost (src/quadstd.cc:4367-4388).
#pragma once

#include <cmath>
#include <vector>

namespace h3dg {

constexpr int kMaxOrder = 10;          // MAX_ELEMENT_ORDER (src/shapeset/common.h:184)
constexpr int kMaxQuadPoints = 13;     // MAX_QUAD_ORDER 24 -> 13 points (src/order.h:27)

inline void legendre_all(int n, long double x, long double *P) {
	P[0] = 1.0L;
	if (n >= 1) P[1] = x;
	for (int k = 1; k < n; k++) P[k + 1] = ((2 * k + 1) * x * P[k] - k * P[k - 1]) / (k + 1);
}

// value of the k-th Lobatto function at x
inline double lobatto_value(int k, double x) {
	if (k == 0) return (1.0 - x) * 0.5;
	if (k == 1) return (1.0 + x) * 0.5;
	long double P[kMaxOrder + 3];
	legendre_all(k, x, P);
	return (double) ((P[k] - P[k - 2]) / sqrtl(2.0L * (2 * k - 1)));
}

// derivative of the k-th Lobatto function at x
inline double lobatto_deriv(int k, double x) {
	if (k == 0) return -0.5;
	if (k == 1) return 0.5;
	long double P[kMaxOrder + 3];
	legendre_all(k - 1, x, P);
	return (double) (sqrtl((2.0L * k - 1) / 2.0L) * P[k - 1]);
}

// n-point Gauss-Legendre rule on [-1, 1], ascending points
inline void gauss_legendre(int n, std::vector<double> &pts, std::vector<double> &wts) {
	pts.assign(n, 0.0);
	wts.assign(n, 0.0);
	const long double pi = 3.141592653589793238462643383279502884L;
	for (int i = 0; i < (n + 1) / 2; i++) {
		long double x = cosl(pi * (i + 0.75L) / (n + 0.5L));
		long double dp = 0;
		for (int it = 0; it < 100; it++) {
			long double p0 = 1, p1 = x;
			for (int k = 1; k < n; k++) {
				long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
				p0 = p1;
				p1 = p2;
			}
			if (n == 1) { p1 = x; p0 = 1; }
			dp = n * (x * p1 - p0) / (x * x - 1);
			long double dx = p1 / dp;
			x -= dx;
			if (fabsl(dx) < 1e-19L) break;
		}
		{
			long double p0 = 1, p1 = x;
			for (int k = 1; k < n; k++) {
				long double p2 = ((2 * k + 1) * x * p1 - k * p0) / (k + 1);
				p0 = p1;
				p1 = p2;
			}
			if (n == 1) { p1 = x; p0 = 1; }
			dp = n * (x * p1 - p0) / (x * x - 1);
		}
		long double w = 2.0L / ((1 - x * x) * dp * dp);
		// x is the i-th largest root; mirror it so the rule is exactly symmetric
		int hi = n - 1 - i, lo = i;
		pts[hi] = (double) x;
		pts[lo] = -(double) x;
		wts[hi] = wts[lo] = (double) w;
	}
	if (n % 2 == 1) pts[n / 2] = 0.0;
}

} // namespace h3dg
