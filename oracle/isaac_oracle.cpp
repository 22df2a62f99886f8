// ISAAC in-situ rendering hot path: CPU restatement used as the parity ORACLE.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product (isaac_b200/) links, loads or
// calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg do, and only as the checker / the timed CPU reference.
//
// Parity status: UNPINNED.  The reference (ComputationalRadiationPhysics/isaac
// 1.7.0) cannot be compiled here (alpaka, Boost, glm, IceT, MPI, jansson and
// libjpeg are absent) and it ships no tests, golden vectors or fixtures.  This
// file restates the reference algorithm function by function, in the same
// operation order, compiled with -ffp-contract=off so that no multiply-add is
// fused (the reference's CPU backend compiled for baseline x86-64 has no FMA).
// Known-answer tests derived by hand from the reference text pin the parser,
// transfer LUT, dither masks, HSV colours and Halton sequence.
//
// glm (pinned by the reference's INSTALL.md to commit 6ad79aae, "0.9.9.9-dev")
// is not vendored; its published semantics are restated here:
//   min(a,b) = b<a ? b : a ; max(a,b) = a<b ? b : a ; clamp = min(max(x,lo),hi)
//   fract(x) = x - floor(x) ; round = half away from zero
//   dot(vec3) = (x*x'+y*y')+z*z' ; dot(vec4) = (x*x'+y*y')+(z*z'+w*w')
//   normalize(v) = v * (1/sqrt(dot(v,v))) ; length(v) = sqrt(dot(v,v))
//   mat4*vec4 = (c0*v.x + c1*v.y) + (c2*v.z + c3*v.w)
//   mat4*mat4 column j = ((A0*B[j][0] + A1*B[j][1]) + A2*B[j][2]) + A3*B[j][3]
//   inverse(mat4) = glm's cofactor expansion (compute_inverse<4,4>)
//
// Every routine is a template over the arithmetic type T: T=float is the
// parity oracle, T=double is the FP64 precision reference.
//
// Reference files cited below are paths inside the ISAAC repository.

#include "../isaac_b200/csrc/isaacb_blue_noise.h"
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc
{
    constexpr int MAX_FUNCTORS = 3; // lib/isaac/isaac_defines.hpp:27-29
    constexpr int MAX_SOURCES = 16; // lib/isaac/isaac_defines.hpp:36-38
    constexpr int MAX_CLIPPING = 16; // lib/isaac/isaac_defines.hpp:44-46
    constexpr int FUNCTOR_COUNT = 6; // idem add mul length pow sum: lib/isaac/isaac_functors.hpp:185-208
    constexpr float Z_NEAR = 0.002f; // lib/isaac/isaac_defines.hpp:53

    enum Op
    {
        OP_IDEM = 0,
        OP_ADD = 1,
        OP_MUL = 2,
        OP_LENGTH = 3,
        OP_POW = 4,
        OP_SUM = 5
    };
    static const char* kFunctorNames[FUNCTOR_COUNT] = {"idem", "add", "mul", "length", "pow", "sum"};

    // ------------------------------------------------------------------ vectors
    template<class T>
    struct V2
    {
        T x, y;
    };
    template<class T>
    struct V3
    {
        T x, y, z;
        T& operator[](int i)
        {
            return (&x)[i];
        }
        const T& operator[](int i) const
        {
            return (&x)[i];
        }
    };
    template<class T>
    struct V4
    {
        T x, y, z, w;
        T& operator[](int i)
        {
            return (&x)[i];
        }
        const T& operator[](int i) const
        {
            return (&x)[i];
        }
    };
    struct I3
    {
        int64_t x, y, z;
        int64_t& operator[](int i)
        {
            return (&x)[i];
        }
        const int64_t& operator[](int i) const
        {
            return (&x)[i];
        }
    };

    template<class T>
    inline T gmin(T a, T b)
    {
        return (b < a) ? b : a;
    }
    template<class T>
    inline T gmax(T a, T b)
    {
        return (a < b) ? b : a;
    }
    template<class T>
    inline T gclamp(T x, T lo, T hi)
    {
        return gmin(gmax(x, lo), hi);
    }
    template<class T>
    inline T gfract(T x)
    {
        return x - std::floor(x);
    }
    template<class T>
    inline T gsign(T x)
    {
        return T((T(0) < x) ? 1 : 0) - T((x < T(0)) ? 1 : 0);
    }

    template<class T>
    inline V3<T> add(V3<T> a, V3<T> b)
    {
        return {a.x + b.x, a.y + b.y, a.z + b.z};
    }
    template<class T>
    inline V3<T> sub(V3<T> a, V3<T> b)
    {
        return {a.x - b.x, a.y - b.y, a.z - b.z};
    }
    template<class T>
    inline V3<T> mul(V3<T> a, V3<T> b)
    {
        return {a.x * b.x, a.y * b.y, a.z * b.z};
    }
    template<class T>
    inline V3<T> muls(V3<T> a, T s)
    {
        return {a.x * s, a.y * s, a.z * s};
    }
    template<class T>
    inline V3<T> smul(T s, V3<T> a)
    {
        return {s * a.x, s * a.y, s * a.z};
    }
    template<class T>
    inline V3<T> divv(V3<T> a, V3<T> b)
    {
        return {a.x / b.x, a.y / b.y, a.z / b.z};
    }
    template<class T>
    inline V3<T> divs(V3<T> a, T s)
    {
        return {a.x / s, a.y / s, a.z / s};
    }
    template<class T>
    inline V3<T> neg(V3<T> a)
    {
        return {-a.x, -a.y, -a.z};
    }
    template<class T>
    inline T dot(V3<T> a, V3<T> b)
    {
        T tx = a.x * b.x, ty = a.y * b.y, tz = a.z * b.z;
        return (tx + ty) + tz;
    }
    template<class T>
    inline T length(V3<T> a)
    {
        return std::sqrt(dot(a, a));
    }
    template<class T>
    inline V3<T> normalize(V3<T> a)
    {
        T inv = T(1) / std::sqrt(dot(a, a));
        return muls(a, inv);
    }

    template<class T>
    inline V4<T> add4(V4<T> a, V4<T> b)
    {
        return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w};
    }
    template<class T>
    inline V4<T> muls4(V4<T> a, T s)
    {
        return {a.x * s, a.y * s, a.z * s, a.w * s};
    }
    template<class T>
    inline V4<T> smul4(T s, V4<T> a)
    {
        return {s * a.x, s * a.y, s * a.z, s * a.w};
    }
    template<class T>
    inline V4<T> divs4(V4<T> a, T s)
    {
        return {a.x / s, a.y / s, a.z / s, a.w / s};
    }

    // Saturating float -> int conversion (the value of a conversion the C++
    // standard leaves undefined; this is the GPU's behaviour and the one the
    // product implements).
    template<class T>
    inline int64_t to_int_sat(T v)
    {
        if(std::isnan(v))
            return 0;
        if(v >= T(2147483647.0))
            return 2147483647;
        if(v <= T(-2147483648.0))
            return -2147483647 - 1;
        return (int64_t)(int32_t) v;
    }

    // transformColor(float4) -> byte4 (lib/isaac/isaac_helper.hpp:71-74): clamp, *255, truncate.
    template<class T>
    inline void to_byte4(V4<T> c, uint8_t* out)
    {
        for(int i = 0; i < 4; ++i)
        {
            T v = gclamp(c[i], T(0), T(1)) * T(255);
            out[i] = (uint8_t) to_int_sat(v);
        }
    }
    // transformColor(byte4) -> float4 (lib/isaac/isaac_helper.hpp:76-79)
    template<class T>
    inline V4<T> from_byte4(const uint8_t* b)
    {
        return {T(b[0]) / T(255), T(b[1]) / T(255), T(b[2]) / T(255), T(b[3]) / T(255)};
    }

    // ------------------------------------------------------------------ mat4 (column major m[c][r])
    template<class T>
    struct M4
    {
        T m[4][4];
    };
    template<class T>
    inline V4<T> mulmv(const M4<T>& M, V4<T> v)
    {
        V4<T> r;
        for(int i = 0; i < 4; ++i)
        {
            T mul0 = M.m[0][i] * v.x;
            T mul1 = M.m[1][i] * v.y;
            T add0 = mul0 + mul1;
            T mul2 = M.m[2][i] * v.z;
            T mul3 = M.m[3][i] * v.w;
            T add1 = mul2 + mul3;
            r[i] = add0 + add1;
        }
        return r;
    }
    template<class T>
    inline M4<T> mulmm(const M4<T>& A, const M4<T>& B)
    {
        M4<T> R;
        for(int c = 0; c < 4; ++c)
            for(int r = 0; r < 4; ++r)
            {
                T s = A.m[0][r] * B.m[c][0];
                s = s + A.m[1][r] * B.m[c][1];
                s = s + A.m[2][r] * B.m[c][2];
                s = s + A.m[3][r] * B.m[c][3];
                R.m[c][r] = s;
            }
        return R;
    }
    // glm compute_inverse<4,4> (cofactor expansion), restated.
    template<class T>
    inline M4<T> inverse(const M4<T>& M)
    {
        auto m = M.m;
        T c00 = m[2][2] * m[3][3] - m[3][2] * m[2][3];
        T c02 = m[1][2] * m[3][3] - m[3][2] * m[1][3];
        T c03 = m[1][2] * m[2][3] - m[2][2] * m[1][3];
        T c04 = m[2][1] * m[3][3] - m[3][1] * m[2][3];
        T c06 = m[1][1] * m[3][3] - m[3][1] * m[1][3];
        T c07 = m[1][1] * m[2][3] - m[2][1] * m[1][3];
        T c08 = m[2][1] * m[3][2] - m[3][1] * m[2][2];
        T c10 = m[1][1] * m[3][2] - m[3][1] * m[1][2];
        T c11 = m[1][1] * m[2][2] - m[2][1] * m[1][2];
        T c12 = m[2][0] * m[3][3] - m[3][0] * m[2][3];
        T c14 = m[1][0] * m[3][3] - m[3][0] * m[1][3];
        T c15 = m[1][0] * m[2][3] - m[2][0] * m[1][3];
        T c16 = m[2][0] * m[3][2] - m[3][0] * m[2][2];
        T c18 = m[1][0] * m[3][2] - m[3][0] * m[1][2];
        T c19 = m[1][0] * m[2][2] - m[2][0] * m[1][2];
        T c20 = m[2][0] * m[3][1] - m[3][0] * m[2][1];
        T c22 = m[1][0] * m[3][1] - m[3][0] * m[1][1];
        T c23 = m[1][0] * m[2][1] - m[2][0] * m[1][1];
        T f0[4] = {c00, c00, c02, c03};
        T f1[4] = {c04, c04, c06, c07};
        T f2[4] = {c08, c08, c10, c11};
        T f3[4] = {c12, c12, c14, c15};
        T f4[4] = {c16, c16, c18, c19};
        T f5[4] = {c20, c20, c22, c23};
        T v0[4] = {m[1][0], m[0][0], m[0][0], m[0][0]};
        T v1[4] = {m[1][1], m[0][1], m[0][1], m[0][1]};
        T v2[4] = {m[1][2], m[0][2], m[0][2], m[0][2]};
        T v3[4] = {m[1][3], m[0][3], m[0][3], m[0][3]};
        T inv0[4], inv1[4], inv2[4], inv3[4];
        for(int i = 0; i < 4; ++i)
        {
            inv0[i] = v1[i] * f0[i] - v2[i] * f1[i] + v3[i] * f2[i];
            inv1[i] = v0[i] * f0[i] - v2[i] * f3[i] + v3[i] * f4[i];
            inv2[i] = v0[i] * f1[i] - v1[i] * f3[i] + v3[i] * f5[i];
            inv3[i] = v0[i] * f2[i] - v1[i] * f4[i] + v2[i] * f5[i];
        }
        const T signA[4] = {T(1), T(-1), T(1), T(-1)};
        const T signB[4] = {T(-1), T(1), T(-1), T(1)};
        M4<T> I;
        for(int i = 0; i < 4; ++i)
        {
            I.m[0][i] = inv0[i] * signA[i];
            I.m[1][i] = inv1[i] * signB[i];
            I.m[2][i] = inv2[i] * signA[i];
            I.m[3][i] = inv3[i] * signB[i];
        }
        T row0[4] = {I.m[0][0], I.m[1][0], I.m[2][0], I.m[3][0]};
        T dot0[4];
        for(int i = 0; i < 4; ++i)
            dot0[i] = m[0][i] * row0[i];
        T dot1 = (dot0[0] + dot0[1]) + (dot0[2] + dot0[3]);
        T oneOverDet = T(1) / dot1;
        for(int c = 0; c < 4; ++c)
            for(int r = 0; r < 4; ++r)
                I.m[c][r] = I.m[c][r] * oneOverDet;
        return I;
    }

    // ------------------------------------------------------------------ helpers (lib/isaac/isaac_helper.hpp)
    // halton (isaac_helper.hpp:57-69)
    inline float halton(uint32_t index, uint32_t base)
    {
        float result = 0;
        float f = 1;
        while(index > 0)
        {
            f /= float(base);
            result += f * float(index % base);
            index /= base;
        }
        return result;
    }

    // getHSVA (isaac_helper.hpp:221-264); h is an isaac_float, M_PI a double.
    inline V4<float> getHSVA(float h, float s, float v, float a)
    {
        int hi = int(std::floor(double(h) / (M_PI / 3)));
        float f = float(double(h) / (M_PI / 3) - double(float(hi)));
        float p = v * (float(1) - s);
        float q = v * (float(1) - s * f);
        float t = v * (float(1) - s * (float(1) - f));
        V4<float> r = {0, 0, 0, a};
        switch(hi)
        {
        case 0:
        case 6:
            r.x = v;
            r.y = t;
            r.z = p;
            break;
        case 1:
            r.x = q;
            r.y = v;
            r.z = p;
            break;
        case 2:
            r.x = p;
            r.y = v;
            r.z = t;
            break;
        case 3:
            r.x = p;
            r.y = q;
            r.z = v;
            break;
        case 4:
            r.x = t;
            r.y = p;
            r.z = v;
            break;
        case 5:
            r.x = v;
            r.y = p;
            r.z = q;
            break;
        }
        return r;
    }

    // ------------------------------------------------------------------ functor chain
    // Host parser: the per-source body of IsaacVisualization::updateFunctions
    // (lib/isaac.hpp:1084-1186).  Returns the reference's errorCode.  Parameter
    // slots the reference leaves indeterminate (a number that fails to parse)
    // are zero here.
    inline int parse_chain(const std::string& text, int bytecode[MAX_FUNCTORS], float params[4 * MAX_FUNCTORS])
    {
        int errorCode = 0;
        std::string source = text;
        size_t pos = 0;
        bool again = true;
        int elem = 0;
        for(int i = 0; i < 4 * MAX_FUNCTORS; ++i)
            params[i] = 0.0f;
        while(again && ((pos = source.find("|")) != std::string::npos || ((again = false) == false)))
        {
            if(elem >= MAX_FUNCTORS)
            {
                errorCode = 1;
                break;
            }
            std::string token = source.substr(0, pos);
            source.erase(0, pos + 1);
            token.erase(
                std::remove_if(token.begin(), token.end(), [](unsigned char c) { return std::isspace(c) != 0; }),
                token.end());
            size_t tBegin = token.find("(");
            float* p = params + 4 * elem;
            if(tBegin == std::string::npos)
            {
                p[0] = p[1] = p[2] = p[3] = 0.0f;
            }
            else
            {
                size_t tEnd = token.find(")");
                if(tEnd == std::string::npos)
                {
                    errorCode = -1;
                    break;
                }
                if(tEnd - tBegin == 1)
                {
                    p[0] = p[1] = p[2] = p[3] = 0.0f;
                }
                else
                {
                    std::string parameters = token.substr(tBegin + 1, tEnd - tBegin - 1);
                    size_t pPos = 0;
                    bool pAgain = true;
                    int pElem = 0;
                    while(pAgain
                          && ((pPos = parameters.find(",")) != std::string::npos || ((pAgain = false) == false)))
                    {
                        if(pElem >= 4)
                        {
                            errorCode = 2;
                            break;
                        }
                        std::string par = parameters.substr(0, pPos);
                        parameters.erase(0, pPos + 1);
                        try
                        {
                            p[pElem] = std::stof(par);
                        }
                        catch(const std::invalid_argument&)
                        {
                            errorCode = -2;
                            pElem++;
                            break;
                        }
                        catch(const std::out_of_range&)
                        {
                            errorCode = -2;
                            pElem++;
                            break;
                        }
                        pElem++;
                    }
                    for(; pElem < 4; pElem++)
                        p[pElem] = p[pElem - 1];
                }
            }
            if(tBegin != std::string::npos)
                token = token.substr(0, tBegin);
            bool found = false;
            for(int f = 0; f < FUNCTOR_COUNT && !found; ++f)
            {
                if(token == kFunctorNames[f])
                {
                    bytecode[elem] = f;
                    found = true;
                }
            }
            if(!found)
            {
                errorCode = -2;
                break;
            }
            elem++;
        }
        for(; elem < MAX_FUNCTORS; elem++)
        {
            bytecode[elem] = 0;
            float* p = params + 4 * elem;
            p[0] = p[1] = p[2] = p[3] = 0.0f;
        }
        return errorCode;
    }

    // glm dot for vec<N>: N=3 (x+y)+z ; N=4 (x+y)+(z+w)
    template<class T>
    inline T dotN(const T* v, int n)
    {
        switch(n)
        {
        case 1:
            return v[0] * v[0];
        case 2:
        {
            T a = v[0] * v[0], b = v[1] * v[1];
            return a + b;
        }
        case 3:
        {
            T a = v[0] * v[0], b = v[1] * v[1], c = v[2] * v[2];
            return (a + b) + c;
        }
        default:
        {
            T a = v[0] * v[0], b = v[1] * v[1], c = v[2] * v[2], d = v[3] * v[3];
            return (a + b) + (c + d);
        }
        }
    }

    // generateFunctorChain (lib/isaac/isaac_functor_chain.hpp:95-108) with the
    // functors of lib/isaac/isaac_functors.hpp:42-183: f2(f1(f0(v,p0),p1),p2).x
    template<class T>
    inline T apply_chain(const T* vin, int dim, const int* bc, const float* params)
    {
        T v[4] = {0, 0, 0, 0};
        for(int i = 0; i < dim; ++i)
            v[i] = vin[i];
        int n = dim;
        for(int k = 0; k < MAX_FUNCTORS; ++k)
        {
            const float* p = params + 4 * k;
            switch(bc[k])
            {
            case OP_ADD:
                for(int i = 0; i < n; ++i)
                    v[i] = v[i] + T(p[i]);
                break;
            case OP_MUL:
                for(int i = 0; i < n; ++i)
                    v[i] = v[i] * T(p[i]);
                break;
            case OP_LENGTH:
                v[0] = std::sqrt(dotN(v, n));
                n = 1;
                break;
            case OP_POW:
                for(int i = 0; i < n; ++i)
                    v[i] = std::pow(v[i], T(p[i]));
                break;
            case OP_SUM:
            {
                T r = T(0);
                for(int i = 0; i < n; ++i)
                    r += v[i];
                v[0] = r;
                n = 1;
                break;
            }
            default:
                break;
            }
        }
        return v[0];
    }

    // Transfer-function lookup index: round(v*TS) clamped to [0,TS-1]
    // (lib/isaac/isaac_common_kernel.hpp:589-591).  NaN -> 0.
    template<class T>
    inline int64_t lut_index(T v, int ts)
    {
        T lookup = std::round(v * T(ts));
        T c = gclamp(lookup, T(0), T(ts - 1));
        if(std::isnan(c))
            return 0;
        return (int64_t) c;
    }

    // ------------------------------------------------------------------ dither (lib/isaac/isaac_dither_kernel.hpp:7-329)
    static const uint8_t kDitherMask1[64]
        = {17, 46, 55, 1,  57, 7,  38, 31, 9,  52, 2,  54, 36, 26, 19, 44, 53, 20, 47, 22, 29, 60,
           62, 12, 45, 14, 26, 33, 8,  39, 11, 63, 13, 56, 6,  50, 40, 32, 23, 48, 21, 42, 51, 5,
           61, 3,  34, 27, 41, 10, 30, 37, 4,  35, 15, 59, 49, 24, 43, 18, 25, 64, 58, 16};
    static const uint8_t kDitherMask2[64]
        = {13, 61, 45, 51, 59, 39, 16, 40, 10, 49, 2,  46, 36, 43, 15, 60, 26, 52, 23, 9,  32, 6,
           31, 0,  54, 21, 58, 24, 17, 5,  28, 38, 56, 41, 11, 63, 14, 47, 37, 48, 42, 62, 12, 18,
           3,  35, 50, 44, 19, 1,  20, 34, 29, 25, 57, 4,  22, 8,  33, 53, 30, 55, 27, 7};

    template<class T>
    inline void dither(int mode, int64_t x, int64_t y, int64_t z, V4<T> c, uint8_t* out)
    {
        if(mode == 0)
        {
            for(int i = 0; i < 4; ++i)
            {
                T v = std::round(gclamp(c[i], T(0), T(1)) * T(255));
                out[i] = (uint8_t) to_int_sat(v);
            }
            return;
        }
        T d;
        if(mode == 1 || mode == 2)
        {
            const uint8_t* mask = (mode == 2) ? kDitherMask2 : kDitherMask1;
            d = T(mask[x % 4 + (y % 4) * 4 + (z % 4) * 16]) / T(64);
        }
        else if(mode == 3)
            d = T(kBlueNoise8[x % 8 + (y % 8) * 8 + (z % 8) * 64]) / T(512);
        else
            d = T(kBlueNoise16[x % 16 + (y % 16) * 16 + (z % 16) * 256]) / T(4096);
        for(int i = 0; i < 4; ++i)
        {
            T s = c[i] * T(255);
            int64_t ci = to_int_sat(s);
            ci += (gfract(s) > d) ? 1 : 0;
            out[i] = (uint8_t) gclamp<int64_t>(ci, 0, 255);
        }
    }

    // ------------------------------------------------------------------ bf16 / fp16 round-trip (IEEE RNE)
    inline float round_to_bf16(float f)
    {
        uint32_t u;
        std::memcpy(&u, &f, 4);
        if((u & 0x7f800000u) == 0x7f800000u)
        { // inf / nan
            if(u & 0x007fffffu)
                u |= 0x00400000u;
            u &= 0xffff0000u;
        }
        else
        {
            uint32_t lsb = (u >> 16) & 1u;
            u += 0x7fffu + lsb;
            u &= 0xffff0000u;
        }
        float r;
        std::memcpy(&r, &u, 4);
        return r;
    }
    inline float round_to_fp16(float f)
    {
        // exact IEEE binary16 RNE via double arithmetic on the representable grid
        if(std::isnan(f))
            return f;
        double a = std::fabs((double) f);
        double sgn = std::signbit(f) ? -1.0 : 1.0;
        if(a >= 65520.0)
            return float(sgn * INFINITY);
        double q;
        if(a < std::ldexp(1.0, -14))
            q = std::ldexp(1.0, -24); // subnormal spacing
        else
        {
            int e;
            std::frexp(a, &e); // a = m*2^e, m in [0.5,1)
            q = std::ldexp(1.0, e - 11);
        }
        double n = a / q;
        double r = std::nearbyint(n); // default rounding mode: ties to even
        return float(sgn * r * q);
    }

    // ------------------------------------------------------------------ context
    struct Clip
    {
        float pos[3];
        float nrm[3];
    };

    struct Particles
    {
        const uint32_t* offsets = nullptr; // ncells+1, cell index = x + y*PX + z*PX*PY
        const float* pos = nullptr; // 3 per particle, cell-relative [0,1)
        const float* attr = nullptr; // featureDim per particle
        const float* radius = nullptr; // per particle or null
        float constRadius = 0.f;
    };

    template<class T>
    struct RayT
    {
        V3<T> dir, start, end;
        T startDepth, endDepth;
        bool isClipped;
        V3<T> clippingNormal;
    };

    class Base
    {
    public:
        virtual ~Base() = default;
    };

    template<class T>
    class Ctx : public Base
    {
    public:
        // geometry (SimulationSizeStruct, lib/isaac/isaac_types.hpp:119-131)
        int W, H;
        int64_t globalSize[3], localSize[3], localParticleSize[3];
        int64_t position[3];
        float scale[3];
        int64_t globalSizeScaled[3], localSizeScaled[3], positionScaled[3];
        int64_t maxGlobalSize, maxGlobalSizeScaled;
        int ts;
        int nVol, nPart, nTotal;
        int featureDim[MAX_SOURCES];
        int persistent[MAX_SOURCES];
        int guard[MAX_SOURCES];
        int storage[MAX_SOURCES]; // 0 fp32, 1 bf16, 2 fp16 (per-source renderer textures)

        // state
        const float* src[MAX_SOURCES] = {};
        Particles part[MAX_SOURCES];
        std::string functions[MAX_SOURCES];
        int bytecode[MAX_SOURCES][MAX_FUNCTORS];
        float params[MAX_SOURCES][4 * MAX_FUNCTORS];
        int errorCode[MAX_SOURCES];
        std::vector<V4<T>> lut[MAX_SOURCES];
        float weight[MAX_SOURCES];
        float iso[MAX_SOURCES];
        float step = 0.5f;
        bool interpolation = false;
        bool optimized = true;
        int clipCount = 0;
        Clip clip[MAX_CLIPPING];
        bool aoEnabled = false;
        float aoWeight = 0.5f;
        bool aoFilter = false;
        int renderMode = 0;
        int ditherMode = 1;
        float bg[4] = {0, 0, 0, 0};
        double proj[16], mv[16];

        // field-source advection (lib/isaac.hpp:292-370, 499-562, 1819-1850); defaults of
        // isaac.hpp:606-643.  The reference leaves the advection textures and their guard
        // cells uninitialised; here they start at zero.
        bool field[MAX_SOURCES] = {};
        // advection textures with the guard band of SyncedTexture3DAllocator
        // (isaac.hpp:206-214): ceil((ISAAC_MAX_ADVECTION_STEP_SIZE + 1) / scale) per axis,
        // x fastest over (localSize + 2 * advGuard)
        std::vector<uint8_t> adv[MAX_SOURCES], advBack[MAX_SOURCES];
        bool advectedThisFrame = false; // advectFrame() ran; the next update() skips it
        std::vector<T> noise; // localSize
        float advStepFactor = 1.0f, advHistoryWeight = 0.95f;
        int advSeedPeriod = 1, advSeedTime = 1, seedPoints = 1000;
        int64_t timeStep = 0;
        bool noiseDirty = true;

        // buffers
        std::vector<uint8_t> volTex, isoTex; // localSize, RGBA8, x fastest
        std::vector<T> npTex[MAX_SOURCES]; // non-persistent textures (local+2g)^3
        std::vector<uint8_t> gColor;
        std::vector<T> gDepth, gAo;
        std::vector<V3<T>> gNormal;
        M4<T> invMVP;
        uint64_t volSamples = 0, isoSamples = 0;

        Ctx(int w,
            int h,
            const int* gs,
            const int* ls,
            const int* lps,
            const int* pos,
            const float* sc,
            int transferSize,
            int nvol,
            int npart,
            const int* fdim,
            const int* pers,
            const int* grd)
        {
            W = w;
            H = h;
            for(int i = 0; i < 3; ++i)
            {
                globalSize[i] = gs[i];
                localSize[i] = ls[i];
                localParticleSize[i] = lps[i];
                position[i] = pos[i];
                scale[i] = sc[i];
                // globalSizeScaled = isaac_float3(globalSize) * scale, stored into isaac_size3 (lib/isaac.hpp:659-661)
                globalSizeScaled[i] = (int64_t) (float(gs[i]) * sc[i]);
                localSizeScaled[i] = (int64_t) (float(ls[i]) * sc[i]);
                positionScaled[i] = (int64_t) (int32_t) (float(pos[i]) * sc[i]);
            }
            maxGlobalSize = std::max(globalSize[0], std::max(globalSize[1], globalSize[2]));
            maxGlobalSizeScaled = std::max(globalSizeScaled[0], std::max(globalSizeScaled[1], globalSizeScaled[2]));
            ts = transferSize;
            nVol = nvol;
            nPart = npart;
            nTotal = nvol + npart;
            for(int i = 0; i < nTotal; ++i)
            {
                featureDim[i] = fdim[i];
                persistent[i] = pers[i];
                guard[i] = grd ? grd[i] : 0;
                storage[i] = 0;
                weight[i] = 2.0f; // ISAAC_DEFAULT_WEIGHT
                iso[i] = 0.0f;
                lut[i].assign(ts, V4<T>{0, 0, 0, 0});
                // default chains (lib/isaac.hpp:720-731): idem for volume and particle sources
                functions[i] = "idem";
                errorCode[i] = parse_chain(functions[i], bytecode[i], params[i]);
                // default transfer functions (lib/isaac.hpp:759-793)
                float hue = float(double(float(2 * i)) * M_PI / double(float(nTotal)));
                std::vector<uint32_t> keys = {0u, (uint32_t) ts};
                V4<float> c0, c1;
                if(i < nVol)
                {
                    c0 = getHSVA(hue, 1, 1, 0);
                    c1 = getHSVA(hue, 1, 1, 1);
                }
                else
                {
                    c0 = getHSVA(hue, 1, 1, 1);
                    c1 = getHSVA(hue, 1, 1, 1);
                }
                float rgba[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
                setTransfer(i, 2, keys.data(), rgba);
            }
            for(int i = 0; i < 16; ++i)
                proj[i] = mv[i] = (i % 5 == 0) ? 1.0 : 0.0;
            volTex.assign(size_t(localSize[0] * localSize[1] * localSize[2]) * 4, 0);
            isoTex.assign(volTex.size(), 0);
            gColor.assign(size_t(W) * H * 4, 0);
            gDepth.assign(size_t(W) * H, 0);
            gAo.assign(size_t(W) * H, 0);
            gNormal.assign(size_t(W) * H, V3<T>{0, 0, 0});
        }

        void setAdvection(float stepFactor, float historyWeight, int period, int seedTime, int seeds)
        {
            advStepFactor = stepFactor;
            advHistoryWeight = historyWeight;
            advSeedPeriod = period;
            advSeedTime = seedTime;
            if(seeds != seedPoints)
                noiseDirty = true;
            seedPoints = seeds;
        }
        int64_t advGuard(int a) const
        {
            return int64_t(std::ceil(float(3 + 1) / scale[a]));
        }
        int64_t advSize(int a) const
        {
            return localSize[a] + 2 * advGuard(a);
        }
        size_t advCount() const
        {
            return size_t(advSize(0) * advSize(1) * advSize(2));
        }
        // index of (x, y, z), each in [-guard, local + guard), in a guarded advection texture
        size_t advIndex(int64_t x, int64_t y, int64_t z) const
        {
            return size_t((x + advGuard(0)) + advSize(0) * ((y + advGuard(1)) + advSize(1) * (z + advGuard(2))));
        }
        void getAdvection(int s, uint8_t* out) const
        {
            const int64_t LX = localSize[0], LY = localSize[1], LZ = localSize[2];
            const bool have = adv[s].size() == advCount();
            for(int64_t z = 0; z < LZ; ++z)
                for(int64_t y = 0; y < LY; ++y)
                    for(int64_t x = 0; x < LX; ++x)
                        out[size_t(x + LX * (y + LY * z))] = have ? adv[s][advIndex(x, y, z)] : 0;
        }

        // direction of neighbour index i (indexToDirection, isaac_types.hpp:133-143)
        static void guardDirection(int i, int d[3])
        {
            for(int a = 0; a < 3; ++a)
            {
                const int m = i % 3;
                d[a] = m == 2 ? -1 : m;
                i /= 3;
            }
        }
        // extent of the guard slab of direction d: guard across it, the local size along it
        void guardSlab(const int d[3], int64_t e[3]) const
        {
            for(int a = 0; a < 3; ++a)
                e[a] = d[a] != 0 ? advGuard(a) : localSize[a];
        }
        // SyncToOwnGuard (isaac_common_kernel.hpp:454-474) on the current advection texture:
        // slab voxel c comes from max(d, 0) * (local - slab - 1) + c per axis
        void packGuard(int s, int i, uint8_t* out) const
        {
            int d[3];
            int64_t e[3];
            guardDirection(i, d);
            guardSlab(d, e);
            for(int64_t z = 0; z < e[2]; ++z)
                for(int64_t y = 0; y < e[1]; ++y)
                    for(int64_t x = 0; x < e[0]; ++x)
                    {
                        const int64_t c[3] = {x, y, z};
                        int64_t src[3];
                        for(int a = 0; a < 3; ++a)
                            src[a] = (d[a] > 0 ? localSize[a] - e[a] - 1 : 0) + c[a];
                        out[size_t(x + e[0] * (y + e[1] * z))] = adv[s][advIndex(src[0], src[1], src[2])];
                    }
        }
        // SyncFromNeighbourGuard (isaac_common_kernel.hpp:477-498): slab voxel c goes to
        // max(d, 0) * (local - 1) + min(d, 0) * slab + c per axis
        void unpackGuard(int s, int i, const uint8_t* in)
        {
            int d[3];
            int64_t e[3];
            guardDirection(i, d);
            guardSlab(d, e);
            for(int64_t z = 0; z < e[2]; ++z)
                for(int64_t y = 0; y < e[1]; ++y)
                    for(int64_t x = 0; x < e[0]; ++x)
                    {
                        const int64_t c[3] = {x, y, z};
                        int64_t dst[3];
                        for(int a = 0; a < 3; ++a)
                            dst[a] = (d[a] > 0 ? localSize[a] - 1 : 0) + (d[a] < 0 ? -e[a] : 0) + c[a];
                        adv[s][advIndex(dst[0], dst[1], dst[2])] = in[size_t(x + e[0] * (y + e[1] * z))];
                    }
        }
        // "advection border" switched off clears both advection textures (isaac.hpp:1668-1683)
        void clearAdvection()
        {
            for(int s = 0; s < nVol; ++s)
            {
                std::fill(adv[s].begin(), adv[s].end(), uint8_t(0));
                std::fill(advBack[s].begin(), advBack[s].end(), uint8_t(0));
            }
        }
        void getNoise(float* out)
        {
            const size_t n = size_t(localSize[0] * localSize[1] * localSize[2]);
            if(noiseDirty || noise.size() != n)
                updateNoise();
            for(size_t i = 0; i < n; ++i)
                out[i] = float(noise[i]);
        }

        void setFramebuffer(int w, int h)
        {
            W = w;
            H = h;
            gColor.assign(size_t(W) * H * 4, 0);
            gDepth.assign(size_t(W) * H, 0);
            gAo.assign(size_t(W) * H, 0);
            gNormal.assign(size_t(W) * H, V3<T>{0, 0, 0});
        }

        // updateTransfer (lib/isaac.hpp:1244-1266) on a description map whose
        // insert keeps the first value of a duplicated key.  Entries outside
        // [first key, last key) keep their previous values.
        void setTransfer(int s, int n, const uint32_t* keys, const float* rgba)
        {
            std::map<uint32_t, V4<float>> desc;
            for(int i = 0; i < n; ++i)
                desc.insert({keys[i], V4<float>{rgba[4 * i], rgba[4 * i + 1], rgba[4 * i + 2], rgba[4 * i + 3]}});
            if(desc.empty())
                return;
            auto next = desc.begin();
            auto before = next;
            for(next++; next != desc.end(); next++)
            {
                uint32_t width = next->first - before->first;
                for(size_t j = 0; j < size_t(width) && size_t(j + before->first) < size_t(ts); j++)
                {
                    T wj = T(float(width - j));
                    T jj = T(float(j));
                    T wf = T(float(width));
                    V4<T> a = {T(before->second.x), T(before->second.y), T(before->second.z), T(before->second.w)};
                    V4<T> b = {T(next->second.x), T(next->second.y), T(next->second.z), T(next->second.w)};
                    V4<T> r;
                    for(int c = 0; c < 4; ++c)
                        r[c] = (a[c] * wj + b[c] * jj) / wf;
                    lut[s][before->first + j] = r;
                }
                before = next;
            }
        }

        int setFunctions(int s, const char* text)
        {
            functions[s] = text;
            errorCode[s] = parse_chain(functions[s], bytecode[s], params[s]);
            return errorCode[s];
        }

        // editClipping (lib/isaac.hpp:956-985)
        bool editClipping(int nr, float px, float py, float pz, float nx, float ny, float nz)
        {
            if(nr >= MAX_CLIPPING || nr < 0)
                return false;
            V3<float> n = {nx, ny, nz};
            V3<float> ns = mul(n, V3<float>{scale[0], scale[1], scale[2]});
            float l = length(ns);
            if(l == 0.0f)
                return false;
            ns = divs(ns, l);
            clip[nr].pos[0] = px;
            clip[nr].pos[1] = py;
            clip[nr].pos[2] = pz;
            clip[nr].nrm[0] = ns.x;
            clip[nr].nrm[1] = ns.y;
            clip[nr].nrm[2] = ns.z;
            return true;
        }
        bool addClipping(float px, float py, float pz, float nx, float ny, float nz)
        {
            if(editClipping(clipCount, px, py, pz, nx, ny, nz))
            {
                clipCount++;
                return true;
            }
            return false;
        }
        void removeClipping(int nr)
        {
            if(nr < 0 || nr >= clipCount)
                return;
            clipCount--;
            for(int i = nr; i < clipCount; i++)
                clip[i] = clip[i + 1];
        }

        // ----- source access (linear x-fastest with guard, featureDim floats per voxel)
        inline void readSource(int s, int64_t x, int64_t y, int64_t z, T* out) const
        {
            int64_t g = guard[s];
            int64_t sx = localSize[0] + 2 * g, sy = localSize[1] + 2 * g;
            size_t idx = size_t((x + g) + (y + g) * sx + (z + g) * sx * sy);
            const float* p = src[s] + idx * featureDim[s];
            for(int c = 0; c < featureDim[s]; ++c)
                out[c] = T(p[c]);
        }
        inline T chainAt(int s, int64_t x, int64_t y, int64_t z) const
        {
            T v[4];
            readSource(s, x, y, z, v);
            return apply_chain<T>(v, featureDim[s], bytecode[s], params[s]);
        }
        inline V4<T> lutAt(int s, T v) const
        {
            return lut[s][lut_index(v, ts)];
        }

        // ----- trilinear sample of a scalar texture (Sampler<LINEAR, ...>::interpolate,
        // lib/isaac/isaac_texture.hpp:237-257, trilinear of isaac_helper.hpp:138-144); fetch(ix, iy, iz)
        // returns the bordered texel
        template<class F>
        T sampleLinear(V3<T> c, F fetch) const
        {
            c = {c.x - T(0.5), c.y - T(0.5), c.z - T(0.5)};
            const int64_t fx = (int64_t) std::floor(c.x), fy = (int64_t) std::floor(c.y), fz = (int64_t) std::floor(c.z);
            T d[2][2][2];
            for(int z = 0; z < 2; ++z)
                for(int y = 0; y < 2; ++y)
                    for(int x = 0; x < 2; ++x)
                        d[x][y][z] = fetch(fx + x, fy + y, fz + z);
            const T ox = gfract(c.x), oy = gfract(c.y), oz = gfract(c.z);
            auto lin = [](T o, T a, T b) { return a * (T(1) - o) + b * o; };
            T a = lin(oy, lin(oz, d[0][0][0], d[0][0][1]), lin(oz, d[0][1][0], d[0][1][1]));
            T b = lin(oy, lin(oz, d[1][0][0], d[1][0][1]), lin(oz, d[1][1][0], d[1][1][1]));
            return lin(ox, a, b);
        }

        // ----- noise texture: HaltonSeedingKernel, three GaussBlur7Kernel passes and
        // MultiplyClampKernel (isaac_common_kernel.hpp:334-430; updateNoiseTexture, isaac.hpp:499-562)
        void updateNoise()
        {
            const int64_t LX = localSize[0], LY = localSize[1], LZ = localSize[2];
            const size_t n = size_t(LX * LY * LZ);
            noise.assign(n, T(0));
            for(uint32_t i = 1; i <= uint32_t(seedPoints); ++i)
            {
                const float ux = halton(i, 3), uy = halton(i, 5), uz = halton(i, 7);
                const int64_t x = (int64_t) (int32_t) (float(LX) * ux), y = (int64_t) (int32_t) (float(LY) * uy),
                              z = (int64_t) (int32_t) (float(LZ) * uz);
                noise[size_t(x + y * LX + z * LX * LY)] = T(1);
            }
            std::vector<T> tmp(n);
            auto blur = [&](const std::vector<T>& src, std::vector<T>& dst, int axis) {
                const T g7[4] = {T(64), T(40.5), T(10), T(1)};
                auto fetch = [&](int64_t x, int64_t y, int64_t z) {
                    // REPEAT border without guard
                    x = (LX + (x % LX)) % LX;
                    y = (LY + (y % LY)) % LY;
                    z = (LZ + (z % LZ)) % LZ;
                    return src[size_t(x + y * LX + z * LX * LY)];
                };
#pragma omp parallel for schedule(static)
                for(int64_t z = 0; z < LZ; ++z)
                    for(int64_t y = 0; y < LY; ++y)
                        for(int64_t x = 0; x < LX; ++x)
                        {
                            T r = T(0);
                            for(int i = -3; i < 4; ++i)
                            {
                                const T mx = axis == 0 ? T(1) : T(0), my = axis == 1 ? T(1) : T(0), mz = axis == 2 ? T(1) : T(0);
                                V3<T> c{T(x) + mx * T(i) / T(scale[0]), T(y) + my * T(i) / T(scale[1]), T(z) + mz * T(i) / T(scale[2])};
                                r += sampleLinear(c, fetch) * g7[i < 0 ? -i : i];
                            }
                            dst[size_t(x + y * LX + z * LX * LY)] = r / T(167);
                        }
            };
            blur(noise, tmp, 0);
            blur(tmp, noise, 1);
            blur(noise, tmp, 2);
            for(size_t i = 0; i < n; ++i)
                noise[i] = gclamp(tmp[i] * T(30), T(0), T(1));
            noiseDirty = false;
        }

        // ----- GenerateAdvectionTextureKernel (isaac_common_kernel.hpp:500-550) for one field source
        void advect(int s)
        {
            const int64_t LX = localSize[0], LY = localSize[1], LZ = localSize[2];
            const T stepSize = T(advStepFactor * float(3)); // ISAAC_MAX_ADVECTION_STEP_SIZE
            const std::vector<uint8_t>& back = advBack[s];
            const int64_t gx = advGuard(0), gy = advGuard(1), gz = advGuard(2);
            auto fetch = [&](int64_t x, int64_t y, int64_t z) {
                // VALUE border (0) outside the guard band (Sampler::safeMemoryAccess,
                // isaac_texture.hpp:201-206); the band holds zeros or a neighbour's slabs
                if(x < -gx || y < -gy || z < -gz || x >= LX + gx || y >= LY + gy || z >= LZ + gz)
                    return T(0);
                return T(back[advIndex(x, y, z)]);
            };
#pragma omp parallel for schedule(static)
            for(int64_t z = 0; z < LZ; ++z)
                for(int64_t y = 0; y < LY; ++y)
                    for(int64_t x = 0; x < LX; ++x)
                    {
                        T v[4];
                        readSource(s, x, y, z, v);
                        V3<T> vec{v[0], v[1], v[2]};
                        const T len = gmax(length(vec), T(std::numeric_limits<float>::min()));
                        vec = {vec.x / len, vec.y / len, vec.z / len};
                        const V3<T> off{vec.x * stepSize / T(scale[0]), vec.y * stepSize / T(scale[1]), vec.z * stepSize / T(scale[2])};
                        const V3<T> oc{(T(x) + T(0.5)) - off.x, (T(y) + T(0.5)) - off.y, (T(z) + T(0.5)) - off.z};
                        const T history = sampleLinear(oc, fetch) / T(255);
                        T nv = noise[size_t(x + y * LX + z * LX * LY)];
                        if(timeStep % advSeedPeriod >= advSeedTime)
                            nv = T(0);
                        V4<T> c{nv + history * T(advHistoryWeight) * (T(1) - nv), T(0), T(0), T(0)};
                        uint8_t out[4];
                        dither(5, x, y, z, c, out);
                        adv[s][advIndex(x, y, z)] = out[0];
                    }
        }

        // ----- per frame: swap the advection buffers, count the step, advect the enabled field sources
        // (isaac.hpp:1819-1850)
        void updateAdvection()
        {
            bool anyField = false;
            for(int s = 0; s < nVol; ++s)
                anyField = anyField || field[s];
            if(!anyField)
                return;
            const size_t n = size_t(localSize[0] * localSize[1] * localSize[2]);
            if(noiseDirty || noise.size() != n)
                updateNoise();
            for(int s = 0; s < nVol; ++s)
            {
                if(!field[s])
                    continue;
                if(adv[s].size() != advCount())
                {
                    adv[s].assign(advCount(), 0);
                    advBack[s].assign(advCount(), 0);
                }
                std::swap(adv[s], advBack[s]);
            }
            timeStep++;
            for(int s = 0; s < nVol; ++s)
                if(field[s] && (weight[s] != 0.0f || iso[s] != 0.0f))
                    advect(s);
        }

        // ----- buffer update: UpdatePersistendTextureKernel (lib/isaac/isaac_common_kernel.hpp:432-451)
        // and MergeToCombinedTextureKernel (lib/isaac/isaac_common_kernel.hpp:690-759).
        // the advection step alone, so that guard slabs can be exchanged before the merge
        void advectFrame()
        {
            updateAdvection();
            advectedThisFrame = true;
        }

        void update()
        {
            if(!advectedThisFrame)
                updateAdvection();
            advectedThisFrame = false;
            for(int s = 0; s < nVol; ++s)
            {
                bool enabled = weight[s] != 0.0f || iso[s] != 0.0f;
                if(!enabled || persistent[s])
                    continue;
                int64_t g = guard[s];
                int64_t sx = localSize[0] + 2 * g, sy = localSize[1] + 2 * g, sz = localSize[2] + 2 * g;
                npTex[s].assign(size_t(sx * sy * sz), T(0));
#pragma omp parallel for schedule(static)
                for(int64_t z = 0; z < sz; ++z)
                    for(int64_t y = 0; y < sy; ++y)
                        for(int64_t x = 0; x < sx; ++x)
                        {
                            T v = chainAt(s, x - g, y - g, z - g);
                            if(storage[s] == 1)
                                v = T(round_to_bf16(float(v)));
                            else if(storage[s] == 2)
                                v = T(round_to_fp16(float(v)));
                            npTex[s][size_t(x + y * sx + z * sx * sy)] = v;
                        }
            }
            if(!optimized)
                return;
            float totalWeight = 0;
            for(int s = 0; s < nVol; ++s)
                totalWeight += weight[s];
            const int64_t LX = localSize[0], LY = localSize[1], LZ = localSize[2];
#pragma omp parallel for schedule(static)
            for(int64_t z = 0; z < LZ; ++z)
                for(int64_t y = 0; y < LY; ++y)
                    for(int64_t x = 0; x < LX; ++x)
                    {
                        V4<T> vc = {0, 0, 0, 0}, ic = {0, 0, 0, 0};
                        for(int s = 0; s < nVol; ++s)
                        {
                            const T vw = T(weight[s]);
                            const T it = T(iso[s]);
                            if(!(vw + it > T(0)))
                                continue;
                            T texValue = chainAt(s, x, y, z);
                            V4<T> color = lutAt(s, texValue);
                            // field sources: alpha blended with the advection texture
                            // (MergeAdvectionToCombinedTextureIterator, isaac_common_kernel.hpp:664-665)
                            if(field[s])
                                color.w *= (T(adv[s][advIndex(x, y, z)]) / T(255));
                            if(vw > T(0))
                            {
                                V4<T> c = color;
                                c.w *= vw;
                                c.x *= c.w;
                                c.y *= c.w;
                                c.z *= c.w;
                                vc = add4(vc, c);
                            }
                            if(it > T(0))
                            {
                                V4<T> c = color;
                                c.w = c.w / it * T(0.5);
                                if(ic.w < c.w)
                                    ic = c;
                            }
                        }
                        vc = divs4(vc, T(totalWeight));
                        size_t o = size_t(x + y * LX + z * LX * LY) * 4;
                        dither(ditherMode, x, y, z, vc, &volTex[o]);
                        for(int c = 0; c < 4; ++c)
                        {
                            T v = std::round(gclamp(ic[c], T(0), T(1)) * T(255));
                            isoTex[o + c] = (uint8_t) to_int_sat(v);
                        }
                    }
        }

        // ----- min/max: MinMaxKernel + CalcMinMaxIterator (lib/isaac/isaac_min_max_kernel.hpp:22-60,
        // lib/isaac.hpp:372-434) and the particle variants (isaac_min_max_kernel.hpp:63-97, isaac.hpp:437-497)
        void minmax(float* mn, float* mx)
        {
            for(int s = 0; s < nTotal; ++s)
            {
                bool isPart = s >= nVol;
                const int64_t* L = isPart ? localParticleSize : localSize;
                int64_t ncol = L[0] * L[1];
                std::vector<T> cmin(size_t(std::max<int64_t>(ncol, 0))), cmax(cmin.size());
#pragma omp parallel for schedule(static)
                for(int64_t col = 0; col < ncol; ++col)
                {
                    int64_t x = col % L[0], y = col / L[0];
                    T lo = std::numeric_limits<float>::max();
                    T hi = -std::numeric_limits<float>::max();
                    for(int64_t z = 0; z < L[2]; ++z)
                    {
                        if(!isPart)
                        {
                            T v = chainAt(s, x, y, z);
                            lo = gmin(lo, v);
                            hi = gmax(hi, v);
                        }
                        else
                        {
                            const Particles& P = part[s];
                            int64_t cell = x + y * L[0] + z * L[0] * L[1];
                            for(uint32_t k = P.offsets[cell]; k < P.offsets[cell + 1]; ++k)
                            {
                                T a[4];
                                for(int c = 0; c < featureDim[s]; ++c)
                                    a[c] = T(P.attr[size_t(k) * featureDim[s] + c]);
                                T v = apply_chain<T>(a, featureDim[s], bytecode[s], params[s]);
                                lo = gmin(lo, v);
                                hi = gmax(hi, v);
                            }
                        }
                    }
                    cmin[col] = lo;
                    cmax[col] = hi;
                }
                T lo = std::numeric_limits<float>::max();
                T hi = -std::numeric_limits<float>::max();
                for(int64_t i = 0; i < ncol; ++i)
                {
                    if(cmin[i] < lo)
                        lo = cmin[i];
                    if(cmax[i] > hi)
                        hi = cmax[i];
                }
                mn[s] = float(lo);
                mx[s] = float(hi);
            }
        }

        // ----- ray setup: pixelToRay / clipRay (lib/isaac/isaac_common_kernel.hpp:51-193)
        RayT<T> pixelToRay(int64_t px, int64_t py) const
        {
            V2<T> vp = {T(px) / T(W) * T(2) - T(1), T(py) / T(H) * T(2) - T(1)};
            V4<T> s4 = mulmv(invMVP, V4<T>{vp.x, vp.y, T(-1), T(1)});
            V4<T> e4 = mulmv(invMVP, V4<T>{vp.x, vp.y, T(1), T(1)});
            RayT<T> r;
            r.start = {s4.x / s4.w, s4.y / s4.w, s4.z / s4.w};
            r.end = {e4.x / e4.w, e4.y / e4.w, e4.z / e4.w};
            T maxSize = T(float(maxGlobalSizeScaled)) * T(0.5);
            r.start = muls(r.start, maxSize);
            r.end = muls(r.end, maxSize);
            r.dir = normalize(sub(r.end, r.start));
            r.isClipped = false;
            r.clippingNormal = {0, 0, 0};
            return r;
        }

        bool clipRay(RayT<T>& ray) const
        {
            V3<T> cpos[MAX_CLIPPING], cnrm[MAX_CLIPPING];
            V3<T> gss = {T(float(globalSizeScaled[0])), T(float(globalSizeScaled[1])), T(float(globalSizeScaled[2]))};
            for(int i = 0; i < clipCount; ++i)
            {
                V3<T> p = {T(clip[i].pos[0]), T(clip[i].pos[1]), T(clip[i].pos[2])};
                cpos[i] = muls(mul(p, gss), T(0.5));
                cnrm[i] = {T(clip[i].nrm[0]), T(clip[i].nrm[1]), T(clip[i].nrm[2])};
            }
            V3<T> off;
            for(int i = 0; i < 3; ++i)
                off[i] = T(float(int32_t(globalSizeScaled[i]) / 2 - int32_t(positionScaled[i])));
            ray.start = add(ray.start, off);
            ray.end = add(ray.end, off);
            for(int i = 0; i < clipCount; ++i)
                cpos[i] = add(cpos[i], off);
            V3<T> bbMin, bbMax;
            for(int i = 0; i < 3; ++i)
            {
                int32_t mnl = std::max<int32_t>(0, -int32_t(positionScaled[i]));
                int32_t mxl = std::min<int32_t>(
                    int32_t(localSizeScaled[i]),
                    int32_t(globalSizeScaled[i]) - int32_t(positionScaled[i]));
                bbMin[i] = (T(float(mnl)) - ray.start[i]) / ray.dir[i];
                bbMax[i] = (T(float(mxl)) - ray.start[i]) / ray.dir[i];
                if(bbMax[i] < bbMin[i])
                    std::swap(bbMax[i], bbMin[i]);
            }
            ray.startDepth = gmax(bbMin.x, gmax(bbMin.y, bbMin.z));
            ray.endDepth = gmin(bbMax.x, gmin(bbMax.y, bbMax.z));
            for(int i = 0; i < 3; ++i)
            {
                T sign = gsign(ray.dir[i]);
                bool outerLow = position[i] == 0 && (sign + T(1)) != T(0);
                bool outerHigh = position[i] + localSize[i] == globalSize[i] && (sign - T(1)) != T(0);
                if(bbMin[i] == ray.startDepth && (outerLow || outerHigh))
                {
                    ray.isClipped = true;
                    ray.clippingNormal[i] = sign;
                }
            }
            for(int i = 0; i < clipCount; ++i)
            {
                T d = dot(ray.dir, cnrm[i]);
                T depth = (dot(cpos[i], cnrm[i]) - dot(ray.start, cnrm[i])) / d;
                if(d > T(0))
                {
                    if(ray.endDepth < depth)
                        return false;
                    if(ray.startDepth <= depth)
                    {
                        ray.clippingNormal = cnrm[i];
                        ray.isClipped = true;
                        ray.startDepth = depth;
                    }
                }
                else
                {
                    if(ray.startDepth > depth)
                        return false;
                    if(ray.endDepth > depth)
                        ray.endDepth = depth;
                }
            }
            ray.startDepth = gmax(ray.startDepth, T(Z_NEAR));
            if(ray.startDepth > ray.endDepth || std::isinf(ray.startDepth) || std::isinf(ray.endDepth))
                return false;
            return true;
        }

        // ----- combined texture sampler: Sampler<filter, CLAMP, normalized=true> on Tex3D<byte4>
        // (lib/isaac/isaac_texture.hpp:140-305)
        inline V4<T> texelB(const std::vector<uint8_t>& tex, int64_t x, int64_t y, int64_t z) const
        {
            x = gclamp<int64_t>(x, 0, localSize[0] - 1);
            y = gclamp<int64_t>(y, 0, localSize[1] - 1);
            z = gclamp<int64_t>(z, 0, localSize[2] - 1);
            const uint8_t* p = &tex[size_t(x + y * localSize[0] + z * localSize[0] * localSize[1]) * 4];
            return {T(p[0]), T(p[1]), T(p[2]), T(p[3])};
        }
        template<class V>
        static inline V lerpv(T o, const V& a, const V& b);

        inline V4<T> sampleB(const std::vector<uint8_t>& tex, V3<T> c) const
        {
            V4<T> r;
            if(interpolation)
            {
                c = {c.x - T(0.5), c.y - T(0.5), c.z - T(0.5)};
                int64_t fx = (int64_t) std::floor(c.x), fy = (int64_t) std::floor(c.y),
                        fz = (int64_t) std::floor(c.z);
                V4<T> d[2][2][2];
                for(int z = 0; z < 2; ++z)
                    for(int y = 0; y < 2; ++y)
                        for(int x = 0; x < 2; ++x)
                            d[x][y][z] = texelB(tex, fx + x, fy + y, fz + z);
                V3<T> f = {gfract(c.x), gfract(c.y), gfract(c.z)};
                r = trilinear4(f, d);
            }
            else
            {
                r = texelB(tex, (int64_t) c.x, (int64_t) c.y, (int64_t) c.z);
            }
            return divs4(r, T(255));
        }

        // linear/bilinear/trilinear (lib/isaac/isaac_helper.hpp:124-144): z first, then y, then x
        static inline V4<T> lin4(T o, V4<T> a, V4<T> b)
        {
            T om = T(1) - o;
            V4<T> r;
            for(int i = 0; i < 4; ++i)
                r[i] = a[i] * om + b[i] * o;
            return r;
        }
        static inline V4<T> trilinear4(V3<T> f, V4<T> (&d)[2][2][2])
        {
            V4<T> a0 = lin4(f.z, d[0][0][0], d[0][0][1]);
            V4<T> b0 = lin4(f.z, d[0][1][0], d[0][1][1]);
            V4<T> A = lin4(f.y, a0, b0);
            V4<T> a1 = lin4(f.z, d[1][0][0], d[1][0][1]);
            V4<T> b1 = lin4(f.z, d[1][1][0], d[1][1][1]);
            V4<T> B = lin4(f.y, a1, b1);
            return lin4(f.x, A, B);
        }
        static inline T lin1(T o, T a, T b)
        {
            return a * (T(1) - o) + b * o;
        }
        static inline T trilinear1(V3<T> f, T (&d)[2][2][2])
        {
            T A = lin1(f.y, lin1(f.z, d[0][0][0], d[0][0][1]), lin1(f.z, d[0][1][0], d[0][1][1]));
            T B = lin1(f.y, lin1(f.z, d[1][0][0], d[1][0][1]), lin1(f.z, d[1][1][0], d[1][1][1]));
            return lin1(f.x, A, B);
        }

        // ----- per-source sample for the legacy renderer: getColorValue
        // (lib/isaac/isaac_volume_kernel.hpp:101-168)
        V4<T> getColorValue(int s, V3<T> pos) const
        {
            T result;
            if(persistent[s])
            {
                int fd = featureDim[s];
                T data[4] = {0, 0, 0, 0};
                if(!interpolation)
                {
                    readSource(s, (int32_t) pos.x, (int32_t) pos.y, (int32_t) pos.z, data);
                }
                else
                {
                    V3<T> off = {pos.x - T(0.5), pos.y - T(0.5), pos.z - T(0.5)};
                    T d8[4][2][2][2];
                    int32_t ox = (int32_t) off.x, oy = (int32_t) off.y, oz = (int32_t) off.z;
                    for(int x = 0; x < 2; ++x)
                        for(int y = 0; y < 2; ++y)
                            for(int z = 0; z < 2; ++z)
                            {
                                int32_t cx = ox + x, cy = oy + y, cz = oz + z;
                                if(guard[s] < 1)
                                {
                                    if(uint64_t(uint32_t(cx)) >= uint64_t(localSize[0]))
                                        cx = ox + 1 - x;
                                    if(uint64_t(uint32_t(cy)) >= uint64_t(localSize[1]))
                                        cy = oy + 1 - y;
                                    if(uint64_t(uint32_t(cz)) >= uint64_t(localSize[2]))
                                        cz = oz + 1 - z;
                                }
                                T v[4];
                                readSource(s, cx, cy, cz, v);
                                for(int c = 0; c < fd; ++c)
                                    d8[c][x][y][z] = v[c];
                            }
                    V3<T> f = {gfract(off.x), gfract(off.y), gfract(off.z)};
                    for(int c = 0; c < fd; ++c)
                        data[c] = trilinear1(f, d8[c]);
                }
                result = apply_chain<T>(data, fd, bytecode[s], params[s]);
            }
            else
            {
                // Sampler<filter, CLAMP> on the FP32 texture with guard
                int64_t g = guard[s];
                int64_t sx = localSize[0] + 2 * g, sy = localSize[1] + 2 * g, sz = localSize[2] + 2 * g;
                auto texel = [&](int64_t x, int64_t y, int64_t z) -> T {
                    x = gclamp<int64_t>(x + g, 0, sx - 1);
                    y = gclamp<int64_t>(y + g, 0, sy - 1);
                    z = gclamp<int64_t>(z + g, 0, sz - 1);
                    return npTex[s][size_t(x + y * sx + z * sx * sy)];
                };
                if(interpolation)
                {
                    V3<T> c = {pos.x - T(0.5), pos.y - T(0.5), pos.z - T(0.5)};
                    int64_t fx = (int64_t) std::floor(c.x), fy = (int64_t) std::floor(c.y),
                            fz = (int64_t) std::floor(c.z);
                    T d8[2][2][2];
                    for(int z = 0; z < 2; ++z)
                        for(int y = 0; y < 2; ++y)
                            for(int x = 0; x < 2; ++x)
                                d8[x][y][z] = texel(fx + x, fy + y, fz + z);
                    V3<T> f = {gfract(c.x), gfract(c.y), gfract(c.z)};
                    result = trilinear1(f, d8);
                }
                else
                {
                    result = texel((int32_t) pos.x, (int32_t) pos.y, (int32_t) pos.z);
                }
            }
            return lutAt(s, result);
        }

        // checkCoord (lib/isaac/isaac_volume_kernel.hpp:206-214)
        V3<T> checkCoord(int s, V3<T> c) const
        {
            V3<T> r;
            for(int i = 0; i < 3; ++i)
            {
                // -guardSize is computed on an unsigned size_t in the reference
                T lo = guard[s] == 0 ? T(0) : T(float(uint64_t(0) - uint64_t(guard[s])));
                T hi = T(float(localSize[i] + guard[s] - 1)) - T(std::numeric_limits<float>::min());
                r[i] = gclamp(c[i], lo, hi);
            }
            return r;
        }
        V4<T> accessorValue(int s, V3<T> pos) const
        {
            if(persistent[s])
                pos = checkCoord(s, pos);
            return getColorValue(s, pos);
        }

        // ----- kernels (one call per pixel)
        size_t pix(int64_t x, int64_t y) const
        {
            return size_t(x + y * W);
        }

        // ClearBufferKernel (lib/isaac/isaac_common_kernel.hpp:195-217), background swizzle lib/isaac.hpp:2245-2249
        void clearPixel(int64_t x, int64_t y)
        {
            V4<T> bgc = {T(bg[3]), T(bg[2]), T(bg[1]), T(0)};
            to_byte4(bgc, &gColor[pix(x, y) * 4]);
            gNormal[pix(x, y)] = {0, 0, 0};
            gDepth[pix(x, y)] = T(std::numeric_limits<float>::max());
            gAo[pix(x, y)] = 0;
        }

        // ParticleRenderKernel + MergeParticleSourceIterator (lib/isaac/isaac_particle_kernel.hpp:32-260)
        void particlePixel(int64_t px, int64_t py)
        {
            bool any = false;
            for(int s = nVol; s < nTotal; ++s)
                any |= weight[s] != 0.0f;
            if(!any)
                return;
            RayT<T> ray = pixelToRay(px, py);
            if(!clipRay(ray))
                return;
            ray.endDepth = gmin(ray.endDepth, gDepth[pix(px, py)]);
            V3<T> pscale = {
                T(float(localSizeScaled[0])) / T(float(localParticleSize[0])),
                T(float(localSizeScaled[1])) / T(float(localParticleSize[1])),
                T(float(localSizeScaled[2])) / T(float(localParticleSize[2]))};
            V4<T> pColor = {0, 0, 0, 0};
            T depth = T(std::numeric_limits<float>::max());
            bool hit = false;
            int32_t dirSign[3];
            for(int i = 0; i < 3; ++i)
                dirSign[i] = (int32_t) gsign(ray.dir[i]);
            V3<T> cur = add(ray.start, muls(ray.dir, ray.startDepth));
            uint32_t cell[3];
            for(int i = 0; i < 3; ++i)
            {
                int32_t c = (int32_t) (cur[i] / pscale[i]);
                cell[i] = (uint32_t) gclamp<int32_t>(c, 0, int32_t(localParticleSize[i] - 1));
            }
            T rayLength = ray.endDepth - ray.startDepth;
            T tested = 0;
            V3<T> t, dT;
            for(int i = 0; i < 3; ++i)
            {
                t[i] = ((T(float(cell[i])) + T(float(std::max(dirSign[i], 0)))) * pscale[i] - cur[i]) / ray.dir[i];
                dT[i] = pscale[i] / ray.dir[i] * T(float(dirSign[i]));
            }
            for(int i = 0; i < 3; ++i)
                if(ray.dir[i] == T(0))
                    t[i] = T(std::numeric_limits<float>::max());
            V3<T> pNormal = {0, 0, 0};
            while(uint64_t(cell[0]) < uint64_t(localParticleSize[0]) && uint64_t(cell[1]) < uint64_t(localParticleSize[1])
                  && uint64_t(cell[2]) < uint64_t(localParticleSize[2]) && !hit && tested <= rayLength)
            {
                for(int s = nVol; s < nTotal; ++s)
                {
                    if(weight[s] == 0.0f)
                        continue;
                    const Particles& P = part[s];
                    int64_t ci = int64_t(cell[0]) + int64_t(cell[1]) * localParticleSize[0]
                        + int64_t(cell[2]) * localParticleSize[0] * localParticleSize[1];
                    for(uint32_t k = P.offsets[ci]; k < P.offsets[ci + 1]; ++k)
                    {
                        V3<T> pp = {T(P.pos[3 * size_t(k)]), T(P.pos[3 * size_t(k) + 1]), T(P.pos[3 * size_t(k) + 2])};
                        V3<T> ppos = mul(add(pp, V3<T>{T(float(cell[0])), T(float(cell[1])), T(float(cell[2]))}), pscale);
                        V3<T> L = sub(ppos, cur);
                        T radius = T(P.radius ? P.radius[k] : P.constRadius) * T(weight[s]);
                        T r2 = radius * radius;
                        T tca = dot(L, ray.dir);
                        T d2 = dot(L, L) - tca * tca;
                        if(d2 <= r2)
                        {
                            T thc = std::sqrt(r2 - d2);
                            T t0 = tca - thc;
                            T t1 = tca + thc;
                            if(t1 >= T(0) && t0 < depth)
                            {
                                T a[4];
                                for(int c = 0; c < featureDim[s]; ++c)
                                    a[c] = T(P.attr[size_t(k) * featureDim[s] + c]);
                                T res = apply_chain<T>(a, featureDim[s], bytecode[s], params[s]);
                                V4<T> value = lutAt(s, res);
                                if(value.w >= T(0.5f))
                                {
                                    pColor = value;
                                    depth = t0;
                                    hit = true;
                                    pNormal = sub(add(cur, smul(t0, ray.dir)), ppos);
                                    if(t0 < T(0) && ray.isClipped)
                                        pNormal = neg(ray.clippingNormal);
                                }
                            }
                        }
                    }
                }
                if(t.x < t.y && t.x < t.z)
                {
                    cell[0] += (uint32_t) dirSign[0];
                    tested = t.x;
                    t.x += dT.x;
                }
                else if(t.y < t.x && t.y < t.z)
                {
                    cell[1] += (uint32_t) dirSign[1];
                    tested = t.y;
                    t.y += dT.y;
                }
                else
                {
                    cell[2] += (uint32_t) dirSign[2];
                    tested = t.z;
                    t.z += dT.z;
                }
            }
            if(!hit)
                return;
            pNormal = normalize(pNormal);
            pColor.w = T(1);
            to_byte4(pColor, &gColor[pix(px, py) * 4]);
            gNormal[pix(px, py)] = pNormal;
            gDepth[pix(px, py)] = depth + ray.startDepth;
        }

        // ray-march preamble shared by the volume and iso kernels
        struct March
        {
            T stepU, factor;
            int64_t startSteps, endSteps;
            V3<T> stepVec, startU;
        };
        March marchSetup(const RayT<T>& ray, T weightFactor, bool withWeight) const
        {
            March m;
            V3<T> sc = {T(scale[0]), T(scale[1]), T(scale[2])};
            T minSize = T(float(std::min(int32_t(globalSize[0]), std::min(int32_t(globalSize[1]), int32_t(globalSize[2])))));
            m.stepU = T(step) * (length(ray.dir) / length(divv(ray.dir, sc)));
            m.factor = m.stepU / minSize * T(2.0f);
            if(withWeight)
                m.factor = m.factor * weightFactor;
            m.startSteps = to_int_sat(std::ceil(ray.startDepth / m.stepU));
            m.endSteps = to_int_sat(std::floor(ray.endDepth / m.stepU));
            m.stepVec = divv(smul(m.stepU, ray.dir), sc);
            m.startU = divv(ray.start, sc);
            return m;
        }

        // CombinedIsoRenderKernel (lib/isaac/isaac_iso_kernel.hpp:25-128)
        uint64_t isoPixel(int64_t px, int64_t py)
        {
            RayT<T> ray = pixelToRay(px, py);
            if(!clipRay(ray))
                return 0;
            ray.endDepth = gmin(ray.endDepth, gDepth[pix(px, py)]);
            if(ray.endDepth <= ray.startDepth)
                return 0;
            March m = marchSetup(ray, 0, false);
            V3<T> sc = {T(scale[0]), T(scale[1]), T(scale[2])};
            bool hit = false;
            T depth = ray.endDepth;
            V4<T> hitColor = {0, 0, 0, 0};
            V3<T> hitNormal = {0, 0, 0};
            T oldValue = 0;
            uint64_t n = 0;
            for(int64_t i = m.startSteps; i <= m.endSteps && !hit; i++)
            {
                ++n;
                V3<T> pos = add(m.startU, muls(m.stepVec, T(float(i))));
                bool first = ray.isClipped && i == m.startSteps;
                T t = T(float(i)) * m.stepU;
                T value = sampleB(isoTex, pos).w;
                T tmp = oldValue;
                oldValue = value;
                if(value < T(0.5))
                    continue;
                if(first)
                    depth = ray.startDepth;
                else
                    depth = t + m.stepU * (T(0.5) - tmp) / (value - tmp);
                hit = true;
                V3<T> np = add(ray.start, muls(ray.dir, depth));
                V3<T> pu = divv(np, sc);
                hitColor = sampleB(isoTex, pu);
                hitColor.w = T(1);
                V3<T> g;
                g.x = sampleB(isoTex, add(pu, V3<T>{1, 0, 0})).w - sampleB(isoTex, sub(pu, V3<T>{1, 0, 0})).w;
                g.y = sampleB(isoTex, add(pu, V3<T>{0, 1, 0})).w - sampleB(isoTex, sub(pu, V3<T>{0, 1, 0})).w;
                g.z = sampleB(isoTex, add(pu, V3<T>{0, 0, 1})).w - sampleB(isoTex, sub(pu, V3<T>{0, 0, 1})).w;
                T gl = length(g);
                if(first || gl == T(0))
                {
                    g = ray.clippingNormal;
                    gl = T(1);
                }
                hitNormal = divs(neg(g), gl);
            }
            if(hit)
            {
                to_byte4(hitColor, &gColor[pix(px, py) * 4]);
                gNormal[pix(px, py)] = hitNormal;
                gDepth[pix(px, py)] = depth;
            }
            return n;
        }

        // legacy IsoStepRenderKernel (lib/isaac/isaac_iso_kernel.hpp:463-778)
        uint64_t isoLegacyPixel(int64_t px, int64_t py)
        {
            bool any = false;
            for(int s = 0; s < nVol; ++s)
                any |= iso[s] != 0.0f;
            if(!any)
                return 0;
            RayT<T> ray = pixelToRay(px, py);
            if(!clipRay(ray))
                return 0;
            ray.endDepth = gmin(ray.endDepth, gDepth[pix(px, py)]);
            if(ray.endDepth <= ray.startDepth)
                return 0;
            March m = marchSetup(ray, 0, false);
            legacyBounds(m);
            V3<T> sc = {T(scale[0]), T(scale[1]), T(scale[2])};
            bool hit = false;
            T hitDepth = ray.endDepth;
            V4<T> hitColor = {0, 0, 0, 0};
            V3<T> hitNormal = {0, 0, 0};
            T oldValues[MAX_SOURCES] = {};
            uint64_t n = 0;
            for(int64_t i = m.startSteps; i <= m.endSteps && !hit; i++)
            {
                ++n;
                V3<T> pos = add(m.startU, muls(m.stepVec, T(float(i))));
                bool first = ray.isClipped && i == m.startSteps;
                T t = T(float(i)) * m.stepU;
                for(int s = 0; s < nVol; ++s)
                {
                    if(iso[s] == 0.0f)
                        continue;
                    T value = accessorValue(s, pos).w;
                    T prev = oldValues[s];
                    oldValues[s] = value;
                    T thr = T(iso[s]);
                    if(value < thr)
                        continue;
                    T testDepth;
                    if(first)
                        testDepth = ray.startDepth;
                    else
                        testDepth = t + m.stepU * (thr - prev) / (value - prev);
                    if(testDepth > hitDepth)
                        continue;
                    hitDepth = testDepth;
                    hit = true;
                    V3<T> np = add(ray.start, muls(ray.dir, hitDepth));
                    V3<T> pu = divv(np, sc);
                    hitColor = accessorValue(s, pu);
                    hitColor.w = T(1.0f);
                    V3<T> g;
                    g.x = accessorValue(s, add(pu, V3<T>{1, 0, 0})).w - accessorValue(s, sub(pu, V3<T>{1, 0, 0})).w;
                    g.y = accessorValue(s, add(pu, V3<T>{0, 1, 0})).w - accessorValue(s, sub(pu, V3<T>{0, 1, 0})).w;
                    g.z = accessorValue(s, add(pu, V3<T>{0, 0, 1})).w - accessorValue(s, sub(pu, V3<T>{0, 0, 1})).w;
                    T gl = length(g);
                    if(first)
                    {
                        g = ray.clippingNormal;
                        gl = T(1);
                    }
                    hitNormal = divs(neg(g), gl);
                }
            }
            if(hit)
            {
                to_byte4(hitColor, &gColor[pix(px, py) * 4]);
                gNormal[pix(px, py)] = hitNormal;
                gDepth[pix(px, py)] = hitDepth;
            }
            return n;
        }

        // legacy start/end step adjustment (lib/isaac/isaac_volume_kernel.hpp:362-376)
        void legacyBounds(March& m) const
        {
            auto inside = [&](V3<T> p) {
                for(int i = 0; i < 3; ++i)
                {
                    if(p[i] < T(0))
                        return false;
                    if(p[i] >= T(float(localSize[i])))
                        return false;
                }
                return true;
            };
            V3<T> pos = add(m.startU, muls(m.stepVec, T(float(m.startSteps))));
            while(!inside(pos) && m.startSteps <= m.endSteps)
            {
                m.startSteps++;
                pos = add(m.startU, muls(m.stepVec, T(float(m.startSteps))));
            }
            pos = add(m.startU, muls(m.stepVec, T(float(m.endSteps))));
            while(!inside(pos) && m.startSteps <= m.endSteps)
            {
                m.endSteps--;
                pos = add(m.startU, muls(m.stepVec, T(float(m.endSteps))));
            }
        }

        // SSAOKernel (lib/isaac/isaac_ssao_kernel.hpp:38-184)
        void ssaoPixel(int64_t px, int64_t py)
        {
            const int radius = 10;
            T occ = 0;
            T ref = gDepth[pix(px, py)];
            for(int i = -3; i <= 3; ++i)
                for(int j = -3; j <= 3; ++j)
                {
                    int64_t x = gclamp<int64_t>(px + i * radius, 0, W - 1);
                    int64_t y = gclamp<int64_t>(py + j * radius, 0, H - 1);
                    if(gDepth[pix(x, y)] < ref)
                        occ += T(1.0f);
                }
            gAo[pix(px, py)] = gclamp(occ / T(42.0f), T(0.0f), T(1.0f));
        }

        // SSAOFilterKernel (lib/isaac/isaac_ssao_kernel.hpp:191-230); compiled out by the reference (lib/isaac.hpp:2410-2428)
        void ssaoFilterPixel(int64_t px, int64_t py)
        {
            T depth = gAo[pix(px, py)];
            V4<T> c = from_byte4<T>(&gColor[pix(px, py) * 4]);
            T w = T(aoWeight);
            T f = (T(1.0f) - w) + w * (T(1.0f) - depth);
            V4<T> r = {f * c.x, f * c.y, f * c.z, c.w};
            to_byte4(r, &gColor[pix(px, py) * 4]);
        }

        // ShadingKernel (lib/isaac/isaac_common_kernel.hpp:220-320), rank 0
        void shadePixel(int64_t px, int64_t py)
        {
            uint8_t* gc = &gColor[pix(px, py) * 4];
            V4<T> color = from_byte4<T>(gc);
            V3<T> normal = gNormal[pix(px, py)];
            T aoStrength = T(1) - gAo[pix(px, py)];
            const int mode = renderMode;
            if(mode == 7)
            {
                V4<float> h = getHSVA(halton(0, 3) * float(2 * M_PI), 1, 1, float(color.w));
                color = {T(h.x), T(h.y), T(h.z), T(h.w)};
            }
            if(mode < 3 || mode == 7)
            {
                RayT<T> ray = pixelToRay(px, py);
                V3<T> lightDir = neg(ray.dir);
                T lightFactor = std::fabs(dot(normal, lightDir));
                V3<T> halfVector = normalize(add(neg(ray.dir), lightDir));
                T specular = dot(normal, halfVector);
                specular = T(std::pow((double) specular, 4));
                specular *= T(0.5f);
                if(mode == 1)
                    specular = 0;
                T w = T(aoWeight);
                T aoFactor = ((T(1.0f) - w) + w * aoStrength);
                lightFactor += aoFactor;
                lightFactor *= T(0.5f);
                V4<T> sh;
                sh.x = gmin(color.x * lightFactor + specular, T(1));
                sh.y = gmin(color.y * lightFactor + specular, T(1));
                sh.z = gmin(color.z * lightFactor + specular, T(1));
                sh.w = color.w;
                to_byte4(sh, gc);
                if(mode == 2 || mode == 7)
                    gDepth[pix(px, py)] = 0;
            }
            else if(mode == 3)
            {
                V4<T> b = {T(bg[3]), T(bg[2]), T(bg[1]), color.w};
                to_byte4(b, gc);
            }
            else if(mode == 4)
            {
                V3<T> n = add(muls(normal, T(0.5)), V3<T>{T(0.5), T(0.5), T(0.5)});
                to_byte4(V4<T>{n.x, n.y, n.z, color.w}, gc);
                gDepth[pix(px, py)] = 0;
            }
            else if(mode == 5)
            {
                T d = gDepth[pix(px, py)] / T(float(maxGlobalSizeScaled));
                to_byte4(V4<T>{d, d, d, color.w}, gc);
                gDepth[pix(px, py)] = 0;
            }
            else if(mode == 6)
            {
                T w = T(aoWeight);
                T aoFactor = ((T(1.0f) - w) + w * aoStrength);
                to_byte4(V4<T>{aoFactor, aoFactor, aoFactor, color.w}, gc);
                gDepth[pix(px, py)] = 0;
            }
            else if(mode == 8)
            {
                V4<float> h = getHSVA(halton(0, 3) * float(2 * M_PI), 1, 1, 1);
                to_byte4(V4<T>{T(h.x), T(h.y), T(h.z), T(h.w)}, gc);
                gDepth[pix(px, py)] = 0;
            }
        }

        // CombinedVolumeRenderKernel (lib/isaac/isaac_volume_kernel.hpp:23-88)
        uint64_t volumePixel(int64_t px, int64_t py, float totalWeight)
        {
            RayT<T> ray = pixelToRay(px, py);
            if(!clipRay(ray))
                return 0;
            ray.endDepth = gmin(ray.endDepth, gDepth[pix(px, py)]);
            if(ray.endDepth <= ray.startDepth)
                return 0;
            March m = marchSetup(ray, T(totalWeight), true);
            V4<T> color = {0, 0, 0, 0};
            uint64_t n = 0;
            for(int64_t i = m.startSteps; i <= m.endSteps; i++)
            {
                ++n;
                V3<T> pos = add(m.startU, muls(m.stepVec, T(float(i))));
                V4<T> value = sampleB(volTex, pos);
                value = muls4(value, m.factor);
                T w = T(1) - color.w;
                color = add4(color, smul4(w, value));
                if(color.w > T(0.99))
                    break;
            }
            V4<T> solid = from_byte4<T>(&gColor[pix(px, py) * 4]);
            color = add4(color, smul4(T(1) - color.w, solid));
            to_byte4(color, &gColor[pix(px, py) * 4]);
            return n;
        }

        // legacy VolumeRenderKernel (lib/isaac/isaac_volume_kernel.hpp:302-432), including the
        // reference's accumulator that carries value*factor into the next step.
        uint64_t volumeLegacyPixel(int64_t px, int64_t py)
        {
            bool any = false;
            for(int s = 0; s < nVol; ++s)
                any |= weight[s] != 0.0f;
            if(!any)
                return 0;
            RayT<T> ray = pixelToRay(px, py);
            if(!clipRay(ray))
                return 0;
            ray.endDepth = gmin(ray.endDepth, gDepth[pix(px, py)]);
            if(ray.endDepth <= ray.startDepth)
                return 0;
            March m = marchSetup(ray, 0, false);
            legacyBounds(m);
            V4<T> value = {0, 0, 0, 0};
            V4<T> color = {0, 0, 0, 0};
            uint64_t n = 0;
            for(int64_t i = m.startSteps; i <= m.endSteps; i++)
            {
                ++n;
                V3<T> pos = add(m.startU, muls(m.stepVec, T(float(i))));
                for(int s = 0; s < nVol; ++s)
                {
                    if(weight[s] == 0.0f)
                        continue;
                    V4<T> c = getColorValue(s, pos);
                    c.w *= T(weight[s]);
                    value.x += c.x * c.w;
                    value.y += c.y * c.w;
                    value.z += c.z * c.w;
                    value.w += c.w;
                }
                T oma = T(1) - color.w;
                value = muls4(value, m.factor);
                V4<T> colorAdd = smul4(oma, value);
                color = add4(color, colorAdd);
                if(color.w > T(0.99))
                    break;
            }
            V4<T> solid = from_byte4<T>(&gColor[pix(px, py) * 4]);
            color = add4(color, smul4(T(1) - color.w, solid));
            to_byte4(color, &gColor[pix(px, py) * 4]);
            return n;
        }

        // drawCallBack pipeline (lib/isaac.hpp:2140-2543) for rows [r0, r1)
        void render(uint8_t* out, int r0, int r1)
        {
            r0 = std::max(0, r0);
            r1 = std::min(H, r1);
            M4<T> P, MV;
            for(int c = 0; c < 4; ++c)
                for(int r = 0; r < 4; ++r)
                {
                    P.m[c][r] = T(float(proj[c * 4 + r]));
                    MV.m[c][r] = T(float(mv[c * 4 + r]));
                    if(sizeof(T) == 8)
                    {
                        P.m[c][r] = T(proj[c * 4 + r]);
                        MV.m[c][r] = T(mv[c * 4 + r]);
                    }
                }
            invMVP = inverse(mulmm(P, MV));
            volSamples = 0;
            isoSamples = 0;
            const int64_t w = W;
#pragma omp parallel for schedule(dynamic, 1)
            for(int64_t y = r0; y < r1; ++y)
                for(int64_t x = 0; x < w; ++x)
                {
                    clearPixel(x, y);
                    particlePixel(x, y);
                }
            uint64_t isoN = 0;
            if(optimized)
            {
                bool anyIso = false;
                for(int s = 0; s < nVol; ++s)
                    anyIso |= iso[s] > 0;
                if(anyIso)
                {
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : isoN)
                    for(int64_t y = r0; y < r1; ++y)
                        for(int64_t x = 0; x < w; ++x)
                            isoN += isoPixel(x, y);
                }
            }
            else
            {
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : isoN)
                for(int64_t y = r0; y < r1; ++y)
                    for(int64_t x = 0; x < w; ++x)
                        isoN += isoLegacyPixel(x, y);
            }
            isoSamples = isoN;
            if(aoEnabled && aoWeight > 0.0f)
            {
#pragma omp parallel for schedule(static)
                for(int64_t y = r0; y < r1; ++y)
                    for(int64_t x = 0; x < w; ++x)
                        ssaoPixel(x, y);
                if(aoFilter)
                {
#pragma omp parallel for schedule(static)
                    for(int64_t y = r0; y < r1; ++y)
                        for(int64_t x = 0; x < w; ++x)
                            ssaoFilterPixel(x, y);
                }
            }
#pragma omp parallel for schedule(static)
            for(int64_t y = r0; y < r1; ++y)
                for(int64_t x = 0; x < w; ++x)
                    shadePixel(x, y);
            uint64_t volN = 0;
            if(optimized)
            {
                float totalWeight = 0;
                for(int s = 0; s < nTotal; ++s)
                    totalWeight += weight[s];
                if(totalWeight > 0)
                {
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : volN)
                    for(int64_t y = r0; y < r1; ++y)
                        for(int64_t x = 0; x < w; ++x)
                            volN += volumePixel(x, y, totalWeight);
                }
            }
            else
            {
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : volN)
                for(int64_t y = r0; y < r1; ++y)
                    for(int64_t x = 0; x < w; ++x)
                        volN += volumeLegacyPixel(x, y);
            }
            volSamples = volN;
            if(out)
                std::memcpy(out + size_t(r0) * W * 4, &gColor[size_t(r0) * W * 4], size_t(r1 - r0) * W * 4);
        }
    };

    template<class T>
    Ctx<T>* as(void* p)
    {
        return static_cast<Ctx<T>*>(static_cast<Base*>(p));
    }
} // namespace orc

using namespace orc;

// ------------------------------------------------------------------ C ABI for the test harness
// Every entry point dispatches on the context's precision flag (0 = FP32 oracle, 1 = FP64 reference).
struct OrHandle
{
    int f64;
    Base* ctx;
};

#define OR_DISPATCH(h, CALL)                                                                                          \
    do                                                                                                                \
    {                                                                                                                 \
        if((h)->f64)                                                                                                  \
        {                                                                                                             \
            auto* c = static_cast<Ctx<double>*>((h)->ctx);                                                            \
            CALL;                                                                                                     \
        }                                                                                                             \
        else                                                                                                          \
        {                                                                                                             \
            auto* c = static_cast<Ctx<float>*>((h)->ctx);                                                             \
            CALL;                                                                                                     \
        }                                                                                                             \
    } while(0)

extern "C"
{
    void* or_create(
        int f64,
        int w,
        int h,
        const int* globalSize,
        const int* localSize,
        const int* localParticleSize,
        const int* position,
        const float* scale,
        int transferSize,
        int nVol,
        int nPart,
        const int* featureDim,
        const int* persistent,
        const int* guard)
    {
        if(nVol + nPart > MAX_SOURCES || nVol + nPart <= 0)
            return nullptr;
        OrHandle* hd = new OrHandle;
        hd->f64 = f64;
        if(f64)
            hd->ctx = new Ctx<double>(
                w,
                h,
                globalSize,
                localSize,
                localParticleSize,
                position,
                scale,
                transferSize,
                nVol,
                nPart,
                featureDim,
                persistent,
                guard);
        else
            hd->ctx = new Ctx<float>(
                w,
                h,
                globalSize,
                localSize,
                localParticleSize,
                position,
                scale,
                transferSize,
                nVol,
                nPart,
                featureDim,
                persistent,
                guard);
        return hd;
    }
    void or_destroy(void* p)
    {
        OrHandle* h = (OrHandle*) p;
        delete h->ctx;
        delete h;
    }
    void or_set_source(void* p, int s, const float* data)
    {
        OR_DISPATCH((OrHandle*) p, c->src[s] = data);
    }
    void or_set_storage(void* p, int s, int dtype)
    {
        OR_DISPATCH((OrHandle*) p, c->storage[s] = dtype);
    }
    void or_set_particles(
        void* p,
        int s,
        const uint32_t* offsets,
        const float* pos,
        const float* attr,
        const float* radius,
        float constRadius)
    {
        OR_DISPATCH((OrHandle*) p, {
            c->part[s].offsets = offsets;
            c->part[s].pos = pos;
            c->part[s].attr = attr;
            c->part[s].radius = radius;
            c->part[s].constRadius = constRadius;
        });
    }
    int or_set_functions(void* p, int s, const char* text)
    {
        int r = 0;
        OR_DISPATCH((OrHandle*) p, r = c->setFunctions(s, text));
        return r;
    }
    void or_get_chain(void* p, int s, int* bytecode, float* params)
    {
        OR_DISPATCH((OrHandle*) p, {
            std::memcpy(bytecode, c->bytecode[s], sizeof(int) * MAX_FUNCTORS);
            std::memcpy(params, c->params[s], sizeof(float) * 4 * MAX_FUNCTORS);
        });
    }
    void or_set_transfer(void* p, int s, int n, const uint32_t* keys, const float* rgba)
    {
        OR_DISPATCH((OrHandle*) p, c->setTransfer(s, n, keys, rgba));
    }
    void or_get_lut(void* p, int s, float* out)
    {
        OR_DISPATCH((OrHandle*) p, {
            for(int i = 0; i < c->ts; ++i)
                for(int k = 0; k < 4; ++k)
                    out[4 * i + k] = float(c->lut[s][i][k]);
        });
    }
    void or_set_weight(void* p, int s, float w)
    {
        OR_DISPATCH((OrHandle*) p, c->weight[s] = w);
    }
    void or_set_iso(void* p, int s, float v)
    {
        OR_DISPATCH((OrHandle*) p, c->iso[s] = v);
    }
    void or_set_step(void* p, float v)
    {
        // lib/isaac.hpp:1626-1635: step below 0.01 is raised to 0.01
        OR_DISPATCH((OrHandle*) p, c->step = v < 0.01f ? 0.01f : v);
    }
    void or_set_interpolation(void* p, int v)
    {
        OR_DISPATCH((OrHandle*) p, c->interpolation = v != 0);
    }
    void or_set_optimized(void* p, int v)
    {
        OR_DISPATCH((OrHandle*) p, c->optimized = v != 0);
    }
    int or_add_clipping(void* p, float px, float py, float pz, float nx, float ny, float nz)
    {
        int r = 0;
        OR_DISPATCH((OrHandle*) p, r = c->addClipping(px, py, pz, nx, ny, nz));
        return r;
    }
    int or_edit_clipping(void* p, int nr, float px, float py, float pz, float nx, float ny, float nz)
    {
        int r = 0;
        OR_DISPATCH((OrHandle*) p, r = c->editClipping(nr, px, py, pz, nx, ny, nz));
        return r;
    }
    void or_remove_clipping(void* p, int nr)
    {
        OR_DISPATCH((OrHandle*) p, c->removeClipping(nr));
    }
    void or_set_ao(void* p, int enabled, float weight, int filter)
    {
        OR_DISPATCH((OrHandle*) p, {
            c->aoEnabled = enabled != 0;
            c->aoWeight = weight;
            c->aoFilter = filter != 0;
        });
    }
    void or_set_render_mode(void* p, int m)
    {
        OR_DISPATCH((OrHandle*) p, c->renderMode = m);
    }
    void or_set_dither_mode(void* p, int m)
    {
        OR_DISPATCH((OrHandle*) p, c->ditherMode = m);
    }
    void or_set_background(void* p, const float* bg)
    {
        OR_DISPATCH((OrHandle*) p, std::memcpy(c->bg, bg, sizeof(float) * 4));
    }
    void or_set_camera(void* p, const double* proj, const double* mv)
    {
        OR_DISPATCH((OrHandle*) p, {
            std::memcpy(c->proj, proj, sizeof(double) * 16);
            std::memcpy(c->mv, mv, sizeof(double) * 16);
        });
    }
    // a new framebuffer size (the reference fixes it at construction; this
    // lets one oracle stand in for views of several sizes of the same scene)
    // field sources must be scalar-indexed after every other volume source
    void or_set_field(void* p, int s, int enabled)
    {
        OR_DISPATCH((OrHandle*) p, c->field[s] = enabled != 0);
    }
    void or_set_advection(void* p, float stepFactor, float historyWeight, int period, int seedTime, int seeds)
    {
        OR_DISPATCH((OrHandle*) p, c->setAdvection(stepFactor, historyWeight, period, seedTime, seeds));
    }
    void or_get_advection(void* p, int s, uint8_t* out)
    {
        OR_DISPATCH((OrHandle*) p, c->getAdvection(s, out));
    }
    void or_advect(void* p)
    {
        OR_DISPATCH((OrHandle*) p, c->advectFrame());
    }
    void or_pack_guard(void* p, int s, int direction, uint8_t* out)
    {
        OR_DISPATCH((OrHandle*) p, c->packGuard(s, direction, out));
    }
    void or_unpack_guard(void* p, int s, int direction, const uint8_t* in)
    {
        OR_DISPATCH((OrHandle*) p, c->unpackGuard(s, direction, in));
    }
    void or_clear_advection(void* p)
    {
        OR_DISPATCH((OrHandle*) p, c->clearAdvection());
    }
    void or_get_noise(void* p, float* out)
    {
        OR_DISPATCH((OrHandle*) p, c->getNoise(out));
    }
    void or_set_framebuffer(void* p, int w, int h)
    {
        OR_DISPATCH((OrHandle*) p, c->setFramebuffer(w, h));
    }
    void or_update(void* p)
    {
        OR_DISPATCH((OrHandle*) p, c->update());
    }
    void or_render(void* p, uint8_t* out, int r0, int r1)
    {
        OR_DISPATCH((OrHandle*) p, c->render(out, r0, r1));
    }
    void or_minmax(void* p, float* mn, float* mx)
    {
        OR_DISPATCH((OrHandle*) p, c->minmax(mn, mx));
    }
    void or_get_combined(void* p, uint8_t* vol, uint8_t* iso)
    {
        OR_DISPATCH((OrHandle*) p, {
            if(vol)
                std::memcpy(vol, c->volTex.data(), c->volTex.size());
            if(iso)
                std::memcpy(iso, c->isoTex.data(), c->isoTex.size());
        });
    }
    void or_get_gbuffer(void* p, float* depth, float* normal, float* ao)
    {
        OR_DISPATCH((OrHandle*) p, {
            size_t n = size_t(c->W) * c->H;
            for(size_t i = 0; i < n; ++i)
            {
                if(depth)
                    depth[i] = float(c->gDepth[i]);
                if(ao)
                    ao[i] = float(c->gAo[i]);
                if(normal)
                {
                    normal[3 * i] = float(c->gNormal[i].x);
                    normal[3 * i + 1] = float(c->gNormal[i].y);
                    normal[3 * i + 2] = float(c->gNormal[i].z);
                }
            }
        });
    }
    void or_get_inverse_mvp(void* p, float* out)
    {
        OR_DISPATCH((OrHandle*) p, {
            for(int col = 0; col < 4; ++col)
                for(int r = 0; r < 4; ++r)
                    out[col * 4 + r] = float(c->invMVP.m[col][r]);
        });
    }
    unsigned long long or_volume_samples(void* p)
    {
        unsigned long long r = 0;
        OR_DISPATCH((OrHandle*) p, r = c->volSamples);
        return r;
    }
    unsigned long long or_iso_samples(void* p)
    {
        unsigned long long r = 0;
        OR_DISPATCH((OrHandle*) p, r = c->isoSamples);
        return r;
    }

    // ---- stand-alone functions for known-answer tests
    int or_parse_chain(const char* text, int* bytecode, float* params)
    {
        return parse_chain(std::string(text), bytecode, params);
    }
    float or_apply_chain(const float* v, int dim, const int* bytecode, const float* params)
    {
        return apply_chain<float>(v, dim, bytecode, params);
    }
    void or_dither(int mode, int x, int y, int z, const float* c, uint8_t* out)
    {
        dither<float>(mode, x, y, z, V4<float>{c[0], c[1], c[2], c[3]}, out);
    }
    float or_halton(unsigned index, unsigned base)
    {
        return halton(index, base);
    }
    void or_hsva(float h, float s, float v, float a, float* out)
    {
        V4<float> r = getHSVA(h, s, v, a);
        out[0] = r.x;
        out[1] = r.y;
        out[2] = r.z;
        out[3] = r.w;
    }
    void or_inverse(const float* m, float* out)
    {
        M4<float> M;
        for(int c = 0; c < 4; ++c)
            for(int r = 0; r < 4; ++r)
                M.m[c][r] = m[c * 4 + r];
        M4<float> I = inverse(M);
        for(int c = 0; c < 4; ++c)
            for(int r = 0; r < 4; ++r)
                out[c * 4 + r] = I.m[c][r];
    }
    float or_round_bf16(float f)
    {
        return round_to_bf16(f);
    }
    float or_round_fp16(float f)
    {
        return round_to_fp16(f);
    }
    int or_num_threads()
    {
#ifdef _OPENMP
        return omp_get_max_threads();
#else
        return 1;
#endif
    }
}
