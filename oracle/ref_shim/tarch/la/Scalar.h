#pragma once
namespace tarch { namespace la {
inline int aPowI(int i, int a) { int r = 1; for (int k = 0; k < i; k++) r *= a; return r; }
inline bool greater(double a, double b, double eps = 1e-14) { return a - b > eps; }
inline bool equals(double a, double b, double eps = 1e-14) { return (a - b < eps) && (b - a < eps); }
}}
