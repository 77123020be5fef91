// TEST INFRASTRUCTURE ONLY -- the few ROOT names used by the reference's Wigner d-functions, so that
// they compile without ROOT (std:: equivalents).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <iostream>
typedef double Double_t;
typedef int Int_t;
namespace TMath {
inline double Cos(double x) { return std::cos(x); }
inline double Sin(double x) { return std::sin(x); }
inline double Log(double x) { return std::log(x); }
inline double Exp(double x) { return std::exp(x); }
inline double Abs(double x) { return std::fabs(x); }
inline int Abs(int x) { return std::abs(x); }
inline int Nint(double x) { return (int)std::lround(x); }
inline int Max(int a, int b) { return std::max(a, b); }
inline int Min(int a, int b) { return std::min(a, b); }
}  // namespace TMath
