// Accuracy of the binary32 functions in hdcx/fpmath.h against binary64 libm
// references, over the argument ranges the integrator evaluates them on.
// Prints one line per function: name, samples, max ulp error, violations of
// the bound stated in fpmath.h. Exit status 0 when no bound is violated.
#include "hdcx/fpmath.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>

namespace {

// Distance in binary32 ulps between a and the binary32 rounding of ref.
double ulpError(float a, double ref)
{
    if (std::isnan(a) && std::isnan(ref)) return 0.0;
    if (std::isnan(a) || std::isnan(ref)) return 1e30;
    if (std::isinf(ref) || std::isinf(a)) return (float)ref == a ? 0.0 : 1e30;
    const float r = static_cast<float>(ref);
    if (a == r) return 0.0;
    int32_t ia, ir;
    std::memcpy(&ia, &a, 4);
    std::memcpy(&ir, &r, 4);
    // Map to a monotonic integer line.
    const int64_t la = ia < 0 ? -(int64_t)(ia & 0x7fffffff) : ia;
    const int64_t lr = ir < 0 ? -(int64_t)(ir & 0x7fffffff) : ir;
    return std::fabs(static_cast<double>(la - lr));
}

struct Stat {
    const char* name;
    long samples = 0;
    double maxUlp = 0.0;
    long violations = 0;
    void add(double err, double bound)
    {
        ++samples;
        if (err > maxUlp) maxUlp = err;
        if (err > bound) ++violations;
    }
};

}  // namespace

int main(int argc, char** argv)
{
    const long n = argc > 1 ? std::atol(argv[1]) : 1000000;
    std::mt19937_64 g(20261203);
    std::uniform_real_distribution<float> u01(0.0f, 1.0f);
    Stat sn{"sin"}, cs{"cos"}, ex{"exp"}, lg{"log"}, ac{"acos"}, at{"atan2"}, pw{"pow"}, p5{"pow5"};
    for (long i = 0; i < n; ++i) {
        // sin/cos: angles up to a few turns (phi in [0, 2 pi), theta in [0, pi]).
        const float a = -25.0f + 50.0f * u01(g);
        sn.add(ulpError(hdcx_fp_sin(a), std::sin((double)a)), 1.0);
        cs.add(ulpError(hdcx_fp_cos(a), std::cos((double)a)), 1.0);
        // exp over the binary32 range with normal results.
        const float e = -87.0f + 175.0f * u01(g);
        ex.add(ulpError(hdcx_fp_exp(e), std::exp((double)e)), 1.0);
        // log over normal and subnormal arguments.
        const float l = std::ldexp(1.0f + u01(g), -148 + static_cast<int>(275.0f * u01(g)));
        lg.add(ulpError(hdcx_fp_log(l), std::log((double)l)), 2.0);
        const float c = -1.0f + 2.0f * u01(g);
        ac.add(ulpError(hdcx_fp_acos(c), std::acos((double)c)), 1.0);
        const float y = -1.0f + 2.0f * u01(g), x = -1.0f + 2.0f * u01(g);
        at.add(ulpError(hdcx_fp_atan2(y, x), std::atan2((double)y, (double)x)), 4.0);
        const float b = u01(g) * 4.0f, p = 0.25f + 256.0f * u01(g);
        const double ref = std::pow((double)b, (double)p);
        if (ref > 1e-37 && ref < 1e37)
            pw.add(ulpError(hdcx_fp_pow(b, p), ref), 8.0);
        const float q = -8.0f + 16.0f * u01(g);
        const double q5 = (double)q * q * q * q * q;
        p5.add(ulpError(hdcx_fp_pow5(q), q5), 0.5000001);
    }
    // Special values.
    long special = 0;
    const float inf = INFINITY;
    if (!std::isnan(hdcx_fp_sin(inf))) ++special;
    if (!std::isnan(hdcx_fp_cos(NAN))) ++special;
    if (hdcx_fp_exp(-inf) != 0.0f || hdcx_fp_exp(inf) != inf || hdcx_fp_exp(0.0f) != 1.0f) ++special;
    if (hdcx_fp_log(0.0f) != -inf || !std::isnan(hdcx_fp_log(-1.0f)) || hdcx_fp_log(1.0f) != 0.0f) ++special;
    if (hdcx_fp_pow(0.0f, 2.5f) != 0.0f || hdcx_fp_pow(3.0f, 0.0f) != 1.0f || hdcx_fp_pow(1.0f, 1e30f) != 1.0f) ++special;
    if (hdcx_fp_pow(-3.0f, 2.0f) != 9.0f || !std::isnan(hdcx_fp_pow(-3.0f, 0.5f))) ++special;
    if (hdcx_fp_acos(1.0f) != 0.0f || !std::isnan(hdcx_fp_acos(1.5f))) ++special;
    if (hdcx_fp_atan2(0.0f, -1.0f) != 3.14159265358979323846f || hdcx_fp_atan2(-0.0f, 1.0f) != -0.0f) ++special;
    if (hdcx_fp_sin(0.0f) != 0.0f || hdcx_fp_cos(0.0f) != 1.0f) ++special;
    int bad = special != 0;
    for (const Stat* s : {&sn, &cs, &ex, &lg, &ac, &at, &pw, &p5}) {
        std::printf("%s %ld %.1f %ld\n", s->name, s->samples, s->maxUlp, s->violations);
        if (s->violations) bad = 1;
    }
    std::printf("special %ld\n", special);
    return bad;
}
