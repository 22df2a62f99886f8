// Host side of the C ABI declared in include/isaac_b200.h: context state,
// the functor-chain parser, transfer tables, camera set-up and the launch
// sequence of a frame.  The reference keeps this state in
// IsaacVisualization (lib/isaac.hpp:58-3036).
#include "../../include/isaac_b200.h"
#include "isaacb_internal.h"


#include <algorithm>
#include <cctype>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

using namespace isaacb;

namespace
{
    thread_local std::string g_createError;
}

namespace isaacb
{
    // error slot of calls that have no context (isaacb_last_error(NULL))
    void set_global_error(const std::string& msg)
    {
        g_createError = msg;
    }
} // namespace isaacb

namespace
{
    const char* kFunctorNames[6] = {"idem", "add", "mul", "length", "pow", "sum"};

    // The functor-chain grammar of IsaacVisualization::updateFunctions
    // (lib/isaac.hpp:1084-1186), per source:
    //
    //   chain   := functor { '|' functor }     at most kMaxFunctors functors
    //   functor := name [ '(' args ')' ... ]   whitespace anywhere is ignored;
    //                                          text after the first ')' is ignored
    //   args    := number { ',' number }       at most 4; missing ones repeat the last
    //
    // Status (the reference's errorCode, the last one raised wins):
    //    1  more than kMaxFunctors functors (parsing stops)
    //   -1  '(' without any ')'              (parsing stops)
    //   -2  unknown functor name             (parsing stops) or an argument that is
    //       not a number                     (the functor is still taken)
    //    2  more than four arguments         (the functor is still taken)
    // Functors that were not taken become idem with zero parameters.

    std::vector<std::string> split(const std::string& text, char sep)
    {
        std::vector<std::string> out(1);
        for(const char c : text)
        {
            if(c == sep)
                out.emplace_back();
            else
                out.back().push_back(c);
        }
        return out;
    }

    std::string without_spaces(const std::string& text)
    {
        std::string out;
        for(const char c : text)
            if(!std::isspace(static_cast<unsigned char>(c)))
                out.push_back(c);
        return out;
    }

    // One number as std::stof reads it (leading numeric prefix, range checked).
    bool read_number(const std::string& item, float& out)
    {
        try
        {
            out = std::stof(item);
            return true;
        }
        catch(const std::logic_error&) // invalid_argument and out_of_range
        {
            return false;
        }
    }

    // The argument list between the parentheses into p[0..3]; returns 0, 2 or -2.
    int read_arguments(const std::string& list, float* p)
    {
        const std::vector<std::string> items = split(list, ',');
        int status = 0;
        int taken = 0;
        for(const std::string& item : items)
        {
            if(taken == 4)
            {
                status = 2;
                break;
            }
            const bool ok = read_number(item, p[taken]);
            ++taken;
            if(!ok)
            {
                status = -2;
                break;
            }
        }
        for(int k = taken; k < 4; ++k)
            p[k] = p[k - 1];
        return status;
    }

    int functor_index(const std::string& name)
    {
        for(int f = 0; f < 6; ++f)
            if(name == kFunctorNames[f])
                return f;
        return -1;
    }

    int parse_chain(const std::string& text, int32_t* bytecode, float* params)
    {
        std::fill(bytecode, bytecode + kMaxFunctors, 0);
        std::fill(params, params + 4 * kMaxFunctors, 0.0f);
        int status = 0;
        int taken = 0;
        for(const std::string& piece : split(text, '|'))
        {
            if(taken == kMaxFunctors)
            {
                status = 1;
                break;
            }
            const std::string functor = without_spaces(piece);
            float* p = params + 4 * taken;
            std::string name = functor;
            const size_t open = functor.find('(');
            if(open != std::string::npos)
            {
                const size_t close = functor.find(')');
                if(close == std::string::npos)
                {
                    status = -1;
                    break;
                }
                // "()" leaves the parameters at zero.  A ')' before the '(' leaves
                // the list running to the end of the functor.
                if(close != open + 1)
                {
                    const std::string list
                        = close > open ? functor.substr(open + 1, close - open - 1) : functor.substr(open + 1);
                    const int s = read_arguments(list, p);
                    if(s != 0)
                        status = s;
                }
                name = functor.substr(0, open);
            }
            const int op = functor_index(name);
            if(op < 0)
            {
                std::fill(p, p + 4, 0.0f);
                status = -2;
                break;
            }
            bytecode[taken++] = op;
        }
        return status;
    }

    // getHSVA (lib/isaac/isaac_helper.hpp:221-264)
    void hsva(float h, float s, float v, float a, float* out)
    {
        const int hi = int(std::floor(double(h) / (M_PI / 3)));
        const float f = float(double(h) / (M_PI / 3) - double(float(hi)));
        const float p = v * (1.0f - s);
        const float q = v * (1.0f - s * f);
        const float t = v * (1.0f - s * (1.0f - f));
        float r = 0, g = 0, b = 0;
        switch(hi)
        {
        case 0:
        case 6:
            r = v, g = t, b = p;
            break;
        case 1:
            r = q, g = v, b = p;
            break;
        case 2:
            r = p, g = v, b = t;
            break;
        case 3:
            r = p, g = q, b = v;
            break;
        case 4:
            r = t, g = p, b = v;
            break;
        case 5:
            r = v, g = p, b = q;
            break;
        default:
            break;
        }
        out[0] = r;
        out[1] = g;
        out[2] = b;
        out[3] = a;
    }

    // glm::inverse of a float mat4 (compute_inverse<4,4>, cofactor expansion), column major m[c*4+r]
    void inverse4(const float* in, float* out)
    {
        auto m = [&](int c, int r) { return in[c * 4 + r]; };
        const float c00 = m(2, 2) * m(3, 3) - m(3, 2) * m(2, 3);
        const float c02 = m(1, 2) * m(3, 3) - m(3, 2) * m(1, 3);
        const float c03 = m(1, 2) * m(2, 3) - m(2, 2) * m(1, 3);
        const float c04 = m(2, 1) * m(3, 3) - m(3, 1) * m(2, 3);
        const float c06 = m(1, 1) * m(3, 3) - m(3, 1) * m(1, 3);
        const float c07 = m(1, 1) * m(2, 3) - m(2, 1) * m(1, 3);
        const float c08 = m(2, 1) * m(3, 2) - m(3, 1) * m(2, 2);
        const float c10 = m(1, 1) * m(3, 2) - m(3, 1) * m(1, 2);
        const float c11 = m(1, 1) * m(2, 2) - m(2, 1) * m(1, 2);
        const float c12 = m(2, 0) * m(3, 3) - m(3, 0) * m(2, 3);
        const float c14 = m(1, 0) * m(3, 3) - m(3, 0) * m(1, 3);
        const float c15 = m(1, 0) * m(2, 3) - m(2, 0) * m(1, 3);
        const float c16 = m(2, 0) * m(3, 2) - m(3, 0) * m(2, 2);
        const float c18 = m(1, 0) * m(3, 2) - m(3, 0) * m(1, 2);
        const float c19 = m(1, 0) * m(2, 2) - m(2, 0) * m(1, 2);
        const float c20 = m(2, 0) * m(3, 1) - m(3, 0) * m(2, 1);
        const float c22 = m(1, 0) * m(3, 1) - m(3, 0) * m(1, 1);
        const float c23 = m(1, 0) * m(2, 1) - m(2, 0) * m(1, 1);
        const float f0[4] = {c00, c00, c02, c03}, f1[4] = {c04, c04, c06, c07}, f2[4] = {c08, c08, c10, c11};
        const float f3[4] = {c12, c12, c14, c15}, f4[4] = {c16, c16, c18, c19}, f5[4] = {c20, c20, c22, c23};
        const float v0[4] = {m(1, 0), m(0, 0), m(0, 0), m(0, 0)};
        const float v1[4] = {m(1, 1), m(0, 1), m(0, 1), m(0, 1)};
        const float v2[4] = {m(1, 2), m(0, 2), m(0, 2), m(0, 2)};
        const float v3[4] = {m(1, 3), m(0, 3), m(0, 3), m(0, 3)};
        float I[16];
        const float sa[4] = {1, -1, 1, -1}, sb[4] = {-1, 1, -1, 1};
        for(int i = 0; i < 4; ++i)
        {
            const float i0 = v1[i] * f0[i] - v2[i] * f1[i] + v3[i] * f2[i];
            const float i1 = v0[i] * f0[i] - v2[i] * f3[i] + v3[i] * f4[i];
            const float i2 = v0[i] * f1[i] - v1[i] * f3[i] + v3[i] * f5[i];
            const float i3 = v0[i] * f2[i] - v1[i] * f4[i] + v2[i] * f5[i];
            I[0 * 4 + i] = i0 * sa[i];
            I[1 * 4 + i] = i1 * sb[i];
            I[2 * 4 + i] = i2 * sa[i];
            I[3 * 4 + i] = i3 * sb[i];
        }
        const float d0 = m(0, 0) * I[0 * 4 + 0], d1 = m(0, 1) * I[1 * 4 + 0], d2 = m(0, 2) * I[2 * 4 + 0],
                    d3 = m(0, 3) * I[3 * 4 + 0];
        const float det = (d0 + d1) + (d2 + d3);
        const float inv = 1.0f / det;
        for(int i = 0; i < 16; ++i)
            out[i] = I[i] * inv;
    }

    // glm mat4 * mat4: column j = ((A0*B[j][0] + A1*B[j][1]) + A2*B[j][2]) + A3*B[j][3]
    void mul4(const float* A, const float* B, float* R)
    {
        for(int c = 0; c < 4; ++c)
            for(int r = 0; r < 4; ++r)
            {
                float s = A[0 * 4 + r] * B[c * 4 + 0];
                s = s + A[1 * 4 + r] * B[c * 4 + 1];
                s = s + A[2 * 4 + r] * B[c * 4 + 2];
                s = s + A[3 * 4 + r] * B[c * 4 + 3];
                R[c * 4 + r] = s;
            }
    }
} // namespace

struct isaacb_ctx
{
    isaacb_desc desc{};
    Geom g{};
    int nVol = 0, nPart = 0, nTotal = 0;
    int ts = 1024;
    // steering state
    std::string functions[kMaxSources];
    Chain chain[kMaxSources]{};
    int32_t errorCode[kMaxSources]{};
    std::vector<float> lutHost; // nTotal*ts*4
    bool lutDirty = true;
    float weight[kMaxSources]{};
    float iso[kMaxSources]{};
    int storage[kMaxSources]{};
    float step = 0.5f;
    int interpolation = 0;
    int renderer = ISAACB_RENDERER_COMBINED;
    int clipCount = 0;
    float clipPos[kMaxClip][3]{};
    float clipNrm[kMaxClip][3]{};
    int aoEnabled = 0;
    float aoWeight = 0.5f;
    int aoFilter = 0;
    int aoSamples = 0; // 0: the reference's 7x7 grid
    int8_t aoOffsets[2 * kMaxAoSamples] = {};
    int renderMode = 0;
    int ditherMode = 1;
    float bg[4] = {0, 0, 0, 0};
    double proj[16]{}, mv[16]{};
    bool cameraSet = false;
    const float* src[kMaxSources]{};
    float* compact[kMaxSources]{}; // compact interior copies of guarded sources
    ParticleSrc part[kMaxSources]{};
    bool partSet[kMaxSources]{};
    bool counting = false;
    bool isoWritten = false;
    // device buffers
    float4* lutDev = nullptr;
    float4* lutPre = nullptr; // merge scratch: weighted premultiplied table entries
    float4* psPre = nullptr; // per-source march scratch: the same for the active sources
    float* lutPinned = nullptr;
    cudaEvent_t lutEvent = nullptr;
    uint32_t* volLin = nullptr; // merge scratch: the combined volume, linear RGBA8
    uint4* volQ = nullptr;
    uint32_t* isoAQ = nullptr;
    uint32_t* isoLin = nullptr;
    uint8_t* volFlag = nullptr;
    uint8_t* isoFlag = nullptr;
    void* srcBricks[kMaxSources]{};
    size_t srcBrickBytes[kMaxSources]{};
    uchar4* color = nullptr;
    float* depth = nullptr;
    float* normal = nullptr;
    float* ao = nullptr;
    unsigned long long* counters = nullptr;
    float* mmPartial = nullptr;
    float* mmResult = nullptr;
    unsigned long long* mmKeys = nullptr;
    int32_t* errorFlag = nullptr;
    // count of all-zero bricks of the last merge (device memory); the march reads it and
    // checks brick emptiness only when it is not zero
    unsigned int* emptyDev = nullptr;
    // slot order of the combined textures: -1 per merge from the camera, 0 x, 1 y fastest
    int32_t slotOrder = -1;
    // field-source advection (defaults of lib/isaac.hpp:606-643); the textures start at zero
    bool field[kMaxSources]{};
    uint8_t* adv[kMaxSources]{}; // guarded: (local + 2 * advG) per axis
    uint8_t* advBack[kMaxSources]{};
    int advG[3] = {0, 0, 0}; // guard band: ceil((ISAAC_MAX_ADVECTION_STEP_SIZE + 1) / scale) per axis
    bool advectedThisFrame = false; // isaacb_advect ran; the next update merges without advecting
    float* noise = nullptr;
    float* noiseTmp = nullptr;
    bool noiseDirty = true;
    float advStepFactor = 1.0f, advHistoryWeight = 0.95f;
    int advSeedPeriod = 1, advSeedTime = 1, seedPoints = 1000;
    long long timeStep = 0;
    uint32_t updateLaunches = 0, renderLaunches = 0;
    bool timing = false;
    cudaEvent_t ev[2 * ISAACB_TIMING_SLOTS]{};
    bool evUsed[ISAACB_TIMING_SLOTS]{};
    std::string lastError;
};

namespace
{
    isaacb_status fail(isaacb_ctx* c, isaacb_status st, const std::string& msg)
    {
        if(c)
            c->lastError = msg;
        else
            g_createError = msg;
        return st;
    }

    isaacb_status cuda_fail(isaacb_ctx* c, cudaError_t e, const char* what)
    {
        const bool oom = e == cudaErrorMemoryAllocation;
        std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
        return fail(c, oom ? ISAACB_OOM : ISAACB_CUDA_ERROR, m);
    }

#define ISAACB_CUDA(c, call, what)                                                                                    \
    do                                                                                                                \
    {                                                                                                                 \
        cudaError_t e_ = (call);                                                                                      \
        if(e_ != cudaSuccess)                                                                                         \
            return cuda_fail((c), e_, (what));                                                                        \
    } while(0)

    bool valid_src(const isaacb_ctx* c, uint32_t s)
    {
        return c && s < uint32_t(c->nTotal);
    }

    // updateTransfer (lib/isaac.hpp:1244-1266) over a description whose repeated
    // keys keep their first value; entries outside [first key, last key) keep
    // their previous values.
    void build_transfer(isaacb_ctx* c, uint32_t s, uint32_t n, const uint32_t* keys, const float* rgba)
    {
        std::map<uint32_t, const float*> desc;
        for(uint32_t i = 0; i < n; ++i)
            desc.insert({keys[i], rgba + 4 * i});
        if(desc.empty())
            return;
        float* lut = c->lutHost.data() + size_t(s) * c->ts * 4;
        auto next = desc.begin();
        auto before = next;
        for(next++; next != desc.end(); next++)
        {
            const uint32_t width = next->first - before->first;
            for(size_t j = 0; j < size_t(width) && size_t(j + before->first) < size_t(c->ts); j++)
            {
                const float wj = float(width - j), jj = float(j), wf = float(width);
                for(int k = 0; k < 4; ++k)
                    lut[(before->first + j) * 4 + k] = (before->second[k] * wj + next->second[k] * jj) / wf;
            }
            before = next;
        }
        c->lutDirty = true;
    }

    isaacb_status upload_lut(isaacb_ctx* c, cudaStream_t st)
    {
        if(!c->lutDirty)
            return ISAACB_OK;
        // the pinned staging buffer may still feed a previous asynchronous copy
        ISAACB_CUDA(c, cudaEventSynchronize(c->lutEvent), "transfer table staging wait");
        std::memcpy(c->lutPinned, c->lutHost.data(), c->lutHost.size() * sizeof(float));
        ISAACB_CUDA(
            c,
            cudaMemcpyAsync(c->lutDev, c->lutPinned, c->lutHost.size() * sizeof(float), cudaMemcpyHostToDevice, st),
            "transfer table upload");
        ISAACB_CUDA(c, cudaEventRecord(c->lutEvent, st), "transfer table event");
        c->lutDirty = false;
        return ISAACB_OK;
    }

    size_t brick_count(const Geom& g)
    {
        return size_t(g.nb[0]) * g.nb[1] * g.nb[2];
    }

    void fill_view(const isaacb_ctx* c, View& v)
    {
        float P[16], MV[16], PM[16];
        for(int i = 0; i < 16; ++i)
        {
            P[i] = float(c->proj[i]);
            MV[i] = float(c->mv[i]);
        }
        mul4(P, MV, PM);
        inverse4(PM, v.inv);
        v.W = int32_t(c->desc.framebuffer[0]);
        v.H = int32_t(c->desc.framebuffer[1]);
        v.scale = make_float3(c->desc.scale[0], c->desc.scale[1], c->desc.scale[2]);
        v.clipCount = c->clipCount;
        for(int i = 0; i < kMaxClip; ++i)
            for(int k = 0; k < 3; ++k)
            {
                v.clipPos[i][k] = c->clipPos[i][k];
                v.clipNrm[i][k] = c->clipNrm[i][k];
            }
    }

    // events around one phase (slot) when timing is on
    struct PhaseTimer
    {
        isaacb_ctx* c;
        int slot;
        cudaStream_t st;
        PhaseTimer(isaacb_ctx* c_, int s_, cudaStream_t st_) : c(c_), slot(s_), st(st_)
        {
            if(c->timing)
            {
                cudaEventRecord(c->ev[2 * slot], st);
                c->evUsed[slot] = true;
            }
        }
        ~PhaseTimer()
        {
            if(c->timing)
                cudaEventRecord(c->ev[2 * slot + 1], st);
        }
    };

    bool any_iso_active(const isaacb_ctx* c)
    {
        for(int s = 0; s < c->nVol; ++s)
            if(c->iso[s] > 0.0f)
                return true;
        return false;
    }
} // namespace

namespace
{

    size_t voxel_count(const isaacb_ctx* c)
    {
        return size_t(c->desc.local_size[0]) * c->desc.local_size[1] * c->desc.local_size[2];
    }

    // bytes of one guarded advection texture
    size_t adv_count(const isaacb_ctx* c)
    {
        size_t n = 1;
        for(int a = 0; a < 3; ++a)
            n *= size_t(c->desc.local_size[a]) + 2 * size_t(c->advG[a]);
        return n;
    }

    // Per update with field sources (lib/isaac.hpp:1819-1850): the noise texture when its
    // seed count changed, the swap of every field source's front and back advection
    // texture, the step counter, and the advection of each enabled field source.
    isaacb_status advect_fields(isaacb_ctx* c, cudaStream_t st)
    {
        bool any = false;
        for(int s = 0; s < c->nVol; ++s)
            any = any || c->field[s];
        if(!any)
            return ISAACB_OK;
        const size_t n = voxel_count(c);
        if(!c->noise)
        {
            ISAACB_CUDA(c, cudaMalloc(&c->noise, n * sizeof(float)), "noise texture");
            ISAACB_CUDA(c, cudaMalloc(&c->noiseTmp, n * sizeof(float)), "noise texture");
            c->noiseDirty = true;
        }
        NoiseParams np{};
        np.LX = int(c->desc.local_size[0]);
        np.LY = int(c->desc.local_size[1]);
        np.LZ = int(c->desc.local_size[2]);
        for(int i = 0; i < 3; ++i)
            np.scale[i] = c->desc.scale[i];
        np.seedPoints = c->seedPoints;
        if(c->noiseDirty)
        {
            launch_noise(np, c->noise, c->noiseTmp, st);
            c->noiseDirty = false;
        }
        for(int s = 0; s < c->nVol; ++s)
        {
            if(!c->field[s])
                continue;
            if(!c->adv[s])
            {
                const size_t na = adv_count(c);
                ISAACB_CUDA(c, cudaMalloc(&c->adv[s], na), "advection texture");
                ISAACB_CUDA(c, cudaMalloc(&c->advBack[s], na), "advection texture");
                ISAACB_CUDA(c, cudaMemsetAsync(c->adv[s], 0, na, st), "advection texture");
                ISAACB_CUDA(c, cudaMemsetAsync(c->advBack[s], 0, na, st), "advection texture");
            }
            std::swap(c->adv[s], c->advBack[s]);
        }
        c->timeStep++;
        for(int s = 0; s < c->nVol; ++s)
        {
            if(!c->field[s] || !(c->weight[s] != 0.0f || c->iso[s] != 0.0f))
                continue;
            AdvectParams ap{};
            ap.field = c->src[s];
            ap.back = c->advBack[s];
            ap.out = c->adv[s];
            ap.noise = c->noise;
            ap.LX = np.LX;
            ap.LY = np.LY;
            ap.LZ = np.LZ;
            for(int a = 0; a < 3; ++a)
                ap.G[a] = c->advG[a];
            for(int i = 0; i < 3; ++i)
                ap.scale[i] = np.scale[i];
            ap.stepSize = c->advStepFactor * 3.0f; // ISAAC_MAX_ADVECTION_STEP_SIZE (isaac_defines.hpp:21)
            ap.historyWeight = c->advHistoryWeight;
            ap.seedNoise = (c->timeStep % c->advSeedPeriod) >= c->advSeedTime ? 0 : 1;
            launch_advect(ap, st);
        }
        ISAACB_CUDA(c, cudaGetLastError(), "advection");
        return ISAACB_OK;
    }

    // one guard slab of field source s between its current advection texture and a
    // device buffer: pack (SyncToOwnGuard) or unpack (SyncFromNeighbourGuard)
    isaacb_status guard_slab(isaacb_ctx* c, uint32_t s, uint32_t direction, uint8_t* slab, bool pack, cudaStream_t stream)
    {
        if(!c || !slab || s >= uint32_t(c->nVol) || direction < 1 || direction > 26)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_pack_guard / isaacb_unpack_guard: bad arguments (direction 1-26)");
        if(!c->field[s] || !c->adv[s])
            return fail(c, ISAACB_NOT_READY, "guard slab: source " + std::to_string(s) + " has no advection texture yet");
        GuardParams g{};
        g.tex = c->adv[s];
        g.slab = slab;
        uint32_t idx = direction;
        for(int a = 0; a < 3; ++a)
        {
            const int m = int(idx % 3);
            idx /= 3;
            g.d[a] = m == 2 ? -1 : m;
            g.L[a] = int(c->desc.local_size[a]);
            g.G[a] = c->advG[a];
            g.e[a] = g.d[a] != 0 ? g.G[a] : g.L[a];
            if(g.d[a] != 0 && g.L[a] < g.G[a] + 1)
                return fail(c, ISAACB_INVALID_ARG, "guard slab: local size smaller than the guard band + 1");
        }
        if(pack)
            launch_pack_guard(g, stream);
        else
            launch_unpack_guard(g, stream);
        ISAACB_CUDA(c, cudaGetLastError(), "guard slab");
        return ISAACB_OK;
    }

    // A source with guard cells is read through a compact copy of its interior: the
    // combined renderer and min/max read only the interior (MergeToCombinedTextureKernel
    // and MinMaxKernel iterate over the local size, lib/isaac/isaac_common_kernel.hpp:
    // 716-719, lib/isaac/isaac_min_max_kernel.hpp:35-38), which is what every kernel
    // here indexes.
    const float* source_data(const isaacb_ctx* c, int s)
    {
        return c->desc.guard_size[s] != 0 ? c->compact[s] : c->src[s];
    }
    isaacb_status compact_guarded(isaacb_ctx* c, cudaStream_t st)
    {
        for(int s = 0; s < c->nVol; ++s)
        {
            const int g = int(c->desc.guard_size[s]);
            if(g == 0 || !c->src[s])
                continue;
            const int fd = int(c->desc.feature_dim[s]);
            if(!c->compact[s])
                ISAACB_CUDA(c, cudaMalloc(&c->compact[s], size_t(c->g.ls[0]) * c->g.ls[1] * c->g.ls[2] * fd * sizeof(float)),
                            "compact source allocation");
            launch_compact_guarded(c->src[s], c->compact[s], c->g.ls[0], c->g.ls[1], c->g.ls[2], g, fd, st);
            ISAACB_CUDA(c, cudaGetLastError(), "compact guarded source");
            c->updateLaunches++;
        }
        return ISAACB_OK;
    }

    // the merge's launch parameters from a context's state (no launch, no stream work)
    // Slot order of the combined textures for the camera of the merge about to run
    // (Geom::yfast).  The ray-march reads a brick's slots in the order the image's pixels
    // walk the volume: x fastest suits views whose image x axis stays close to the volume's
    // x axis, y fastest (with warps of 4 x 8 pixels) views about the y axis seen from the
    // side, whose image columns follow y.  Measured over an orbit about y at 20 degrees of
    // pitch on 4 x 512^3 sources (a 2.5 GB texture), the two orders cross at 45 degrees of
    // yaw (|image x . volume x| = 0.71); on a 0.33 GB texture (256^3) y fastest was 1 %
    // slower at 94 degrees, as L2 then holds much of the texture and the access order
    // matters less, so the automatic choice applies to textures beyond 4x the L2 cache.
    // Only the speed depends on it: both orders hold the same texels.
    int32_t slot_order_for_camera(const isaacb_ctx* c)
    {
        if(c->slotOrder >= 0)
            return c->slotOrder;
        const double textureBytes = double(brick_count(c->g)) * kSlotsPerBrick * sizeof(uint4);
        if(textureBytes < 4.0 * 126.0e6)
            return 0;
        // rows 0 and 1 of the column-major modelview: the image axes in volume coordinates
        const double ix[3] = {c->mv[0], c->mv[4], c->mv[8]}, iy[3] = {c->mv[1], c->mv[5], c->mv[9]};
        const double nx = std::sqrt(ix[0] * ix[0] + ix[1] * ix[1] + ix[2] * ix[2]);
        const double ny = std::sqrt(iy[0] * iy[0] + iy[1] * iy[1] + iy[2] * iy[2]);
        if(!(nx > 0.0) || !(ny > 0.0))
            return 0;
        const double ex = std::fabs(ix[0]) / nx, ey = std::fabs(iy[1]) / ny;
        return ex < 0.7071 && ey > ex ? 1 : 0;
    }

    void prepare_merge(isaacb_ctx* c, MergeParams& p)
    {
        p.g = c->g;
        p.nVol = c->nVol;
        p.ts = c->ts;
        p.ditherMode = c->ditherMode;
        p.writeIso = any_iso_active(c) ? 1 : 0;
        p.lut = c->lutDev;
        p.lutPre = c->lutPre;
        p.totalWeight = 0.0f;
        for(int s = 0; s < c->nVol; ++s)
        {
            p.src[s] = source_data(c, s);
            p.fdim[s] = int32_t(c->desc.feature_dim[s]);
            p.chain[s] = c->chain[s];
            p.chainIdem[s] = (c->chain[s].op[0] == OP_IDEM && c->chain[s].op[1] == OP_IDEM && c->chain[s].op[2] == OP_IDEM) ? 1 : 0;
            p.weight[s] = c->weight[s];
            p.iso[s] = c->iso[s];
            p.totalWeight += c->weight[s];
        }
        {
            // colour sums are finite and >= 0 when every active table entry and weight is
            bool nonneg = p.totalWeight > 0.0f && std::isfinite(p.totalWeight);
            for(int s = 0; s < c->nVol && nonneg; ++s)
            {
                if(!(c->weight[s] > 0.0f))
                {
                    if(c->weight[s] < 0.0f || c->weight[s] != c->weight[s])
                        nonneg = false;
                    continue;
                }
                const float* l = c->lutHost.data() + size_t(s) * c->ts * 4;
                for(size_t k = 0; k < size_t(c->ts) * 4 && nonneg; ++k)
                    nonneg = l[k] >= 0.0f && std::isfinite(l[k]);
            }
            p.nonNegative = nonneg ? 1 : 0;
        }
        {
            int e2 = 0;
            const float m = std::frexp(p.totalWeight, &e2);
            // an exact power of two whose reciprocal is a normal float
            p.invTotalWeight = (m == 0.5f && e2 > -120 && e2 < 120) ? std::ldexp(1.0f, 1 - e2) : 0.0f;
        }
        p.volLin = c->volLin;
        p.volQ = c->volQ;
        p.isoAQ = c->isoAQ;
        p.isoLin = c->isoLin;
        p.volFlag = c->volFlag;
        p.isoFlag = c->isoFlag;
        p.emptyBricks = c->emptyDev;
        for(int s = 0; s < c->nVol; ++s)
            p.adv[s] = c->field[s] ? c->adv[s] : nullptr;
        for(int a = 0; a < 3; ++a)
            p.advG[a] = c->advG[a];
    }
} // namespace

extern "C"
{
    const char* isaacb_last_error(const isaacb_ctx* ctx)
    {
        return ctx ? ctx->lastError.c_str() : g_createError.c_str();
    }

    isaacb_status isaacb_parse_chain(const char* chain, int32_t* bytecode, float* params, int32_t* error_code)
    {
        if(!chain || !bytecode || !params)
            return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_parse_chain: null argument");
        const int e = parse_chain(std::string(chain), bytecode, params);
        if(error_code)
            *error_code = e;
        return e == 0 ? ISAACB_OK : ISAACB_PARSE_ERROR;
    }

    isaacb_status isaacb_create(const isaacb_desc* d, isaacb_ctx** out)
    {
        if(!d || !out)
            return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: null argument");
        *out = nullptr;
        const uint32_t nTotal = d->n_volume_sources + d->n_particle_sources;
        if(nTotal == 0 || nTotal > uint32_t(kMaxSources))
            return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: 1..16 sources required");
        if(d->framebuffer[0] == 0 || d->framebuffer[1] == 0 || d->framebuffer[0] > 16384 || d->framebuffer[1] > 16384)
            return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: framebuffer must be 1..16384 per side");
        for(int i = 0; i < 3; ++i)
        {
            if(d->local_size[i] == 0 || d->local_size[i] > 8192 || d->global_size[i] == 0 || d->global_size[i] > 1u << 20)
                return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: local/global size out of range");
            if(d->n_particle_sources && (d->local_particle_size[i] == 0 || d->local_particle_size[i] > 8192))
                return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: particle grid out of range");
            if(!(d->scale[i] > 0.0f) || !std::isfinite(d->scale[i]))
                return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: scale must be positive");
        }
        if(d->transfer_size < 2 || d->transfer_size > (1u << 16))
            return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: transfer_size must be 2..65536");
        for(uint32_t s = 0; s < nTotal; ++s)
        {
            if(d->feature_dim[s] < 1 || d->feature_dim[s] > 4)
                return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: feature_dim must be 1..4");
            if(d->guard_size[s] > 64 || (s >= d->n_volume_sources && d->guard_size[s] != 0))
                return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: guard_size must be 0..64 (0 for particle sources)");
        }
        isaacb_ctx* c = new isaacb_ctx;
        c->desc = *d;
        for(int a = 0; a < 3; ++a)
            c->advG[a] = int(std::ceil(float(3 + 1) / d->scale[a])); // isaac.hpp:206-214
        c->nVol = int(d->n_volume_sources);
        c->nPart = int(d->n_particle_sources);
        c->nTotal = int(nTotal);
        c->ts = int(d->transfer_size);
        Geom& g = c->g;
        for(int i = 0; i < 3; ++i)
        {
            g.gs[i] = int32_t(d->global_size[i]);
            g.ls[i] = int32_t(d->local_size[i]);
            g.lps[i] = int32_t(d->local_particle_size[i]);
            g.pos[i] = d->position[i];
            // isaac_float3(size) * scale stored into integer vectors (lib/isaac.hpp:659-661)
            g.gss[i] = int32_t(int64_t(float(d->global_size[i]) * d->scale[i]));
            g.lss[i] = int32_t(int64_t(float(d->local_size[i]) * d->scale[i]));
            g.posS[i] = int32_t(float(d->position[i]) * d->scale[i]);
            g.nb[i] = bricks_per_axis(g.ls[i]);
        }
        g.maxGss = std::max(g.gss[0], std::max(g.gss[1], g.gss[2]));
        if(uint64_t(g.nb[0]) * g.nb[1] * g.nb[2] * kSlotsPerBrick >= (uint64_t(1) << 31))
        {
            delete c;
            return fail(nullptr, ISAACB_INVALID_ARG, "isaacb_create: local volume too large for one context (>~1400^3)");
        }
        // reference defaults (lib/isaac.hpp:720-793)
        c->lutHost.assign(size_t(c->nTotal) * c->ts * 4, 0.0f);
        for(int s = 0; s < c->nTotal; ++s)
        {
            c->weight[s] = 2.0f;
            c->iso[s] = 0.0f;
            c->functions[s] = "idem";
            c->errorCode[s] = parse_chain(c->functions[s], c->chain[s].op, c->chain[s].p);
            const float hue = float(double(float(2 * s)) * M_PI / double(float(c->nTotal)));
            float c0[4], c1[4];
            hsva(hue, 1, 1, s < c->nVol ? 0.0f : 1.0f, c0);
            hsva(hue, 1, 1, 1.0f, c1);
            const uint32_t keys[2] = {0u, uint32_t(c->ts)};
            float rgba[8];
            std::memcpy(rgba, c0, 16);
            std::memcpy(rgba + 4, c1, 16);
            build_transfer(c, uint32_t(s), 2, keys, rgba);
        }
        const size_t npix = size_t(d->framebuffer[0]) * d->framebuffer[1];
        const size_t nbr = brick_count(g);
        cudaError_t e = cudaSuccess;
        auto alloc = [&](void** p, size_t bytes) {
            if(e == cudaSuccess)
                e = cudaMalloc(p, bytes);
        };
        alloc((void**) &c->lutDev, c->lutHost.size() * sizeof(float));
        alloc((void**) &c->lutPre, c->lutHost.size() * sizeof(float));
        alloc((void**) &c->psPre, c->lutHost.size() * sizeof(float));
        if(e == cudaSuccess)
            e = cudaMallocHost((void**) &c->lutPinned, c->lutHost.size() * sizeof(float));
        if(e == cudaSuccess)
            e = cudaEventCreateWithFlags(&c->lutEvent, cudaEventDisableTiming);
        alloc((void**) &c->volQ, nbr * kSlotsPerBrick * sizeof(uint4));
        alloc((void**) &c->isoAQ, nbr * kSlotsPerBrick * sizeof(uint32_t));
        alloc((void**) &c->isoLin, size_t(g.ls[0]) * g.ls[1] * g.ls[2] * sizeof(uint32_t));
        alloc((void**) &c->volLin, size_t(g.ls[0]) * g.ls[1] * g.ls[2] * sizeof(uint32_t));
        alloc((void**) &c->volFlag, nbr);
        alloc((void**) &c->isoFlag, nbr);
        alloc((void**) &c->color, npix * sizeof(uchar4));
        alloc((void**) &c->depth, npix * sizeof(float));
        alloc((void**) &c->normal, npix * 3 * sizeof(float));
        alloc((void**) &c->ao, npix * sizeof(float));
        alloc((void**) &c->counters, 2 * sizeof(unsigned long long));
        alloc((void**) &c->mmPartial, 2 * 148 * 8 * sizeof(float));
        alloc((void**) &c->mmResult, 2 * sizeof(float));
        alloc((void**) &c->mmKeys, 2 * sizeof(unsigned long long));
        alloc((void**) &c->errorFlag, sizeof(int32_t));
        alloc((void**) &c->emptyDev, sizeof(unsigned int));
        if(e == cudaSuccess)
            e = cudaMemset(c->emptyDev, 0, sizeof(unsigned int));
        if(e == cudaSuccess)
            e = cudaMemset(c->errorFlag, 0, sizeof(int32_t));
        if(e == cudaSuccess)
            e = cudaMemset(c->isoLin, 0, size_t(g.ls[0]) * g.ls[1] * g.ls[2] * sizeof(uint32_t));
        if(e == cudaSuccess)
            e = cudaMemset(c->isoFlag, 0, nbr);
        if(e == cudaSuccess)
            e = cudaMemset(c->color, 0, npix * sizeof(uchar4));
        if(e != cudaSuccess)
        {
            const bool oom = e == cudaErrorMemoryAllocation;
            std::string m = std::string("isaacb_create: ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
            isaacb_destroy(c);
            return fail(nullptr, oom ? ISAACB_OOM : ISAACB_CUDA_ERROR, m);
        }
        *out = c;
        return ISAACB_OK;
    }

    isaacb_status isaacb_destroy(isaacb_ctx* c)
    {
        if(!c)
            return ISAACB_OK;
        for(float* q : c->compact)
            cudaFree(q);
        cudaFree(c->lutDev);
        cudaFree(c->lutPre);
        cudaFree(c->psPre);
        if(c->lutPinned)
            cudaFreeHost(c->lutPinned);
        if(c->lutEvent)
            cudaEventDestroy(c->lutEvent);
        cudaFree(c->volQ);
        cudaFree(c->isoAQ);
        cudaFree(c->isoLin);
        cudaFree(c->volLin);
        cudaFree(c->volFlag);
        cudaFree(c->isoFlag);
        for(int s = 0; s < kMaxSources; ++s)
            cudaFree(c->srcBricks[s]);
        cudaFree(c->color);
        cudaFree(c->depth);
        cudaFree(c->normal);
        cudaFree(c->ao);
        cudaFree(c->counters);
        cudaFree(c->mmPartial);
        cudaFree(c->mmResult);
        cudaFree(c->mmKeys);
        cudaFree(c->errorFlag);
        for(int s = 0; s < kMaxSources; ++s)
        {
            cudaFree(c->adv[s]);
            cudaFree(c->advBack[s]);
        }
        cudaFree(c->noise);
        cudaFree(c->noiseTmp);
        cudaFree(c->emptyDev);
        for(auto& e : c->ev)
            if(e)
                cudaEventDestroy(e);
        delete c;
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_source(isaacb_ctx* c, uint32_t s, const float* dev)
    {
        if(!valid_src(c, s) || int(s) >= c->nVol)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_source: not a volume source index");
        c->src[s] = dev;
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_particles(
        isaacb_ctx* c,
        uint32_t s,
        const uint32_t* offsets,
        const float* positions,
        const float* attributes,
        const float* radii,
        float constRadius)
    {
        if(!valid_src(c, s) || int(s) < c->nVol)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_particles: not a particle source index");
        if(!offsets || !positions || !attributes)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_particles: null device pointer");
        ParticleSrc& P = c->part[s - c->nVol];
        P.offsets = offsets;
        P.pos = positions;
        P.attr = attributes;
        P.radius = radii;
        P.constRadius = constRadius;
        c->partSet[s - c->nVol] = true;
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_functions(isaacb_ctx* c, uint32_t s, const char* chain, int32_t* error_code)
    {
        if(!valid_src(c, s) || !chain)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_functions: bad source or null chain");
        c->functions[s] = chain;
        c->errorCode[s] = parse_chain(c->functions[s], c->chain[s].op, c->chain[s].p);
        if(error_code)
            *error_code = c->errorCode[s];
        if(c->errorCode[s] != 0)
            return fail(c, ISAACB_PARSE_ERROR, "isaacb_set_functions: error code " + std::to_string(c->errorCode[s]));
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_transfer(isaacb_ctx* c, uint32_t s, uint32_t n, const uint32_t* keys, const float* rgba)
    {
        if(!valid_src(c, s) || (n && (!keys || !rgba)))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_transfer: bad arguments");
        build_transfer(c, s, n, keys, rgba);
        return ISAACB_OK;
    }

    isaacb_status isaacb_get_transfer(isaacb_ctx* c, uint32_t s, float* lut)
    {
        if(!valid_src(c, s) || !lut)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_get_transfer: bad arguments");
        std::memcpy(lut, c->lutHost.data() + size_t(s) * c->ts * 4, size_t(c->ts) * 4 * sizeof(float));
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_weight(isaacb_ctx* c, uint32_t s, float w)
    {
        if(!valid_src(c, s))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_weight: bad source");
        c->weight[s] = w;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_iso_threshold(isaacb_ctx* c, uint32_t s, float v)
    {
        if(!valid_src(c, s))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_iso_threshold: bad source");
        c->iso[s] = v;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_step(isaacb_ctx* c, float v)
    {
        if(!c || !(v == v))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_step: bad step");
        c->step = v < 0.01f ? 0.01f : v;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_interpolation(isaacb_ctx* c, int32_t v)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        c->interpolation = v != 0;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_renderer(isaacb_ctx* c, int32_t r)
    {
        if(!c || (r != ISAACB_RENDERER_COMBINED && r != ISAACB_RENDERER_PER_SOURCE))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_renderer: unknown renderer");
        c->renderer = r;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_slot_order(isaacb_ctx* c, int32_t order)
    {
        if(!c || order < -1 || order > 1)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_slot_order: order must be -1, 0 or 1");
        c->slotOrder = order;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_storage(isaacb_ctx* c, uint32_t s, int32_t dt)
    {
        if(!valid_src(c, s) || int(s) >= c->nVol || dt < 0 || dt > 2)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_storage: bad source or dtype");
        c->storage[s] = dt;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_ao(isaacb_ctx* c, int32_t enabled, float weight, int32_t filter)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        c->aoEnabled = enabled != 0;
        c->aoWeight = weight;
        c->aoFilter = filter != 0;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_ao_pattern(isaacb_ctx* c, uint32_t samples, float radius)
    {
        if(!c || samples > uint32_t(kMaxAoSamples) || (samples > 0 && !(radius >= 1.0f && radius <= 127.0f)))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_ao_pattern: samples 0..32, radius 1..127 px");
        // a golden-angle spiral filling the disc evenly: tap k at radius r*sqrt((k+0.5)/n),
        // angle k * pi * (3 - sqrt(5)), rounded to whole pixels
        const double golden = 3.14159265358979323846 * (3.0 - std::sqrt(5.0));
        for(uint32_t k = 0; k < samples; ++k)
        {
            const double r = double(radius) * std::sqrt((double(k) + 0.5) / double(samples));
            const double a = golden * double(k);
            c->aoOffsets[2 * k] = int8_t(std::lround(r * std::cos(a)));
            c->aoOffsets[2 * k + 1] = int8_t(std::lround(r * std::sin(a)));
        }
        c->aoSamples = int(samples);
        return ISAACB_OK;
    }
    isaacb_status isaacb_get_ao_pattern(isaacb_ctx* c, uint32_t* samples, int32_t* offsets)
    {
        if(!c || !samples)
            return ISAACB_INVALID_ARG;
        *samples = uint32_t(c->aoSamples);
        if(offsets)
            for(int k = 0; k < 2 * c->aoSamples; ++k)
                offsets[k] = c->aoOffsets[k];
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_render_mode(isaacb_ctx* c, int32_t m)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        c->renderMode = m;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_dither_mode(isaacb_ctx* c, int32_t m)
    {
        // 0 rounding, 1 ordered 4^3, 2 blue noise 4^3, 3 blue noise 8^3, any larger value blue noise 16^3
        if(!c || m < 0)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_dither_mode: mode must be >= 0");
        c->ditherMode = m;
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_field_source(isaacb_ctx* c, uint32_t s, int32_t enabled)
    {
        if(!c || s >= uint32_t(c->nVol))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_field_source: bad source");
        if(enabled && c->desc.feature_dim[s] != 3)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_field_source: a field source is a float3 vector field");
        if(enabled && c->desc.guard_size[s] != 0)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_field_source: field sources take no guard cells here");
        bool f[kMaxSources];
        for(int k = 0; k < c->nVol; ++k)
            f[k] = c->field[k];
        f[s] = enabled != 0;
        // the reference merges the volume sources, then the field sources: field sources
        // must follow every other volume source
        for(int k = 0; k + 1 < c->nVol; ++k)
            if(f[k] && !f[k + 1])
                return fail(c, ISAACB_INVALID_ARG, "isaacb_set_field_source: field sources must be the last volume sources");
        c->field[s] = f[s];
        return ISAACB_OK;
    }
    isaacb_status isaacb_set_advection(
        isaacb_ctx* c,
        float step_factor,
        float history_weight,
        int32_t seeding_period,
        int32_t seeding_duration,
        int32_t seed_points)
    {
        if(!c || seeding_period < 1 || seed_points < 0)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_advection: seeding period >= 1 and seed points >= 0");
        c->advStepFactor = step_factor;
        c->advHistoryWeight = history_weight;
        c->advSeedPeriod = seeding_period;
        c->advSeedTime = seeding_duration;
        if(seed_points != c->seedPoints)
            c->noiseDirty = true;
        c->seedPoints = seed_points;
        return ISAACB_OK;
    }
    isaacb_status isaacb_get_advection(isaacb_ctx* c, void* stream, uint32_t s, uint8_t* host)
    {
        if(!c || !host || s >= uint32_t(c->nVol))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_get_advection: bad arguments");
        cudaStream_t st = (cudaStream_t) stream;
        const size_t n = voxel_count(c);
        if(!c->adv[s])
        {
            std::memset(host, 0, n);
            return ISAACB_OK;
        }
        // the interior of the guarded texture
        const size_t LX = c->desc.local_size[0], LY = c->desc.local_size[1], LZ = c->desc.local_size[2];
        const size_t SX = LX + 2 * c->advG[0], SY = LY + 2 * c->advG[1];
        cudaMemcpy3DParms m{};
        m.srcPtr = make_cudaPitchedPtr(c->adv[s], SX, SX, SY);
        m.srcPos = make_cudaPos(size_t(c->advG[0]), size_t(c->advG[1]), size_t(c->advG[2]));
        m.dstPtr = make_cudaPitchedPtr(host, LX, LX, LY);
        m.extent = make_cudaExtent(LX, LY, LZ);
        m.kind = cudaMemcpyDeviceToHost;
        ISAACB_CUDA(c, cudaMemcpy3DAsync(&m, st), "advection readback");
        ISAACB_CUDA(c, cudaStreamSynchronize(st), "advection readback");
        return ISAACB_OK;
    }

    isaacb_status isaacb_advect(isaacb_ctx* c, void* stream)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        for(int s = 0; s < c->nVol; ++s)
            if(c->field[s] && !c->src[s] && (c->weight[s] != 0.0f || c->iso[s] != 0.0f))
                return fail(c, ISAACB_NOT_READY, "isaacb_advect: field source " + std::to_string(s) + " has no memory");
        const isaacb_status r = advect_fields(c, (cudaStream_t) stream);
        if(r != ISAACB_OK)
            return r;
        ISAACB_CUDA(c, cudaGetLastError(), "isaacb_advect");
        c->advectedThisFrame = true;
        return ISAACB_OK;
    }

    isaacb_status isaacb_advection_guard(const isaacb_ctx* c, uint32_t guard[3])
    {
        if(!c || !guard)
            return ISAACB_INVALID_ARG;
        for(int a = 0; a < 3; ++a)
            guard[a] = uint32_t(c->advG[a]);
        return ISAACB_OK;
    }

    isaacb_status isaacb_pack_guard(isaacb_ctx* c, uint32_t s, uint32_t direction, uint8_t* slab, void* stream)
    {
        return guard_slab(c, s, direction, slab, true, (cudaStream_t) stream);
    }

    isaacb_status isaacb_unpack_guard(isaacb_ctx* c, uint32_t s, uint32_t direction, const uint8_t* slab, void* stream)
    {
        return guard_slab(c, s, direction, const_cast<uint8_t*>(slab), false, (cudaStream_t) stream);
    }

    isaacb_status isaacb_clear_advection(isaacb_ctx* c, void* stream)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        const size_t na = adv_count(c);
        for(int s = 0; s < c->nVol; ++s)
        {
            if(c->adv[s])
                ISAACB_CUDA(c, cudaMemsetAsync(c->adv[s], 0, na, (cudaStream_t) stream), "clear advection");
            if(c->advBack[s])
                ISAACB_CUDA(c, cudaMemsetAsync(c->advBack[s], 0, na, (cudaStream_t) stream), "clear advection");
        }
        return ISAACB_OK;
    }
    isaacb_status isaacb_get_noise(isaacb_ctx* c, void* stream, float* host)
    {
        if(!c || !host)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_get_noise: bad arguments");
        cudaStream_t st = (cudaStream_t) stream;
        const size_t n = voxel_count(c);
        if(!c->noise)
        {
            ISAACB_CUDA(c, cudaMalloc(&c->noise, n * sizeof(float)), "noise texture");
            ISAACB_CUDA(c, cudaMalloc(&c->noiseTmp, n * sizeof(float)), "noise texture");
            c->noiseDirty = true;
        }
        if(c->noiseDirty)
        {
            NoiseParams np{};
            np.LX = int(c->desc.local_size[0]);
            np.LY = int(c->desc.local_size[1]);
            np.LZ = int(c->desc.local_size[2]);
            for(int i = 0; i < 3; ++i)
                np.scale[i] = c->desc.scale[i];
            np.seedPoints = c->seedPoints;
            launch_noise(np, c->noise, c->noiseTmp, st);
            c->noiseDirty = false;
        }
        ISAACB_CUDA(c, cudaMemcpyAsync(host, c->noise, n * sizeof(float), cudaMemcpyDeviceToHost, st), "noise readback");
        ISAACB_CUDA(c, cudaStreamSynchronize(st), "noise readback");
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_background(isaacb_ctx* c, const float* rgba)
    {
        if(!c || !rgba)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_background: null argument");
        std::memcpy(c->bg, rgba, sizeof(c->bg));
        return ISAACB_OK;
    }

    isaacb_status isaacb_edit_clipping(isaacb_ctx* c, uint32_t nr, const float* pos, const float* n)
    {
        if(!c || !pos || !n || nr >= uint32_t(kMaxClip))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_edit_clipping: bad plane index or null argument");
        // editClipping (lib/isaac.hpp:956-985): the normal is scaled and normalised
        float ns[3] = {n[0] * c->desc.scale[0], n[1] * c->desc.scale[1], n[2] * c->desc.scale[2]};
        const float t0 = ns[0] * ns[0], t1 = ns[1] * ns[1], t2 = ns[2] * ns[2];
        const float l = std::sqrt((t0 + t1) + t2);
        if(l == 0.0f)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_edit_clipping: zero normal");
        for(int k = 0; k < 3; ++k)
        {
            c->clipPos[nr][k] = pos[k];
            c->clipNrm[nr][k] = ns[k] / l;
        }
        return ISAACB_OK;
    }
    isaacb_status isaacb_add_clipping(isaacb_ctx* c, const float* pos, const float* n)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        isaacb_status st = isaacb_edit_clipping(c, uint32_t(c->clipCount), pos, n);
        if(st == ISAACB_OK)
            c->clipCount++;
        return st;
    }
    isaacb_status isaacb_remove_clipping(isaacb_ctx* c, uint32_t nr)
    {
        if(!c || nr >= uint32_t(c->clipCount))
            return fail(c, ISAACB_INVALID_ARG, "isaacb_remove_clipping: no such plane");
        c->clipCount--;
        for(int i = int(nr); i < c->clipCount; ++i)
            for(int k = 0; k < 3; ++k)
            {
                c->clipPos[i][k] = c->clipPos[i + 1][k];
                c->clipNrm[i][k] = c->clipNrm[i + 1][k];
            }
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_camera(isaacb_ctx* c, const double* proj, const double* mv)
    {
        if(!c || !proj || !mv)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_set_camera: null argument");
        std::memcpy(c->proj, proj, sizeof(c->proj));
        std::memcpy(c->mv, mv, sizeof(c->mv));
        c->cameraSet = true;
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_counting(isaacb_ctx* c, int32_t on)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        c->counting = on != 0;
        return ISAACB_OK;
    }

    isaacb_status isaacb_update(isaacb_ctx* c, void* stream)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        cudaStream_t st = (cudaStream_t) stream;
        for(int s = 0; s < c->nVol; ++s)
            if(!c->src[s] && (c->weight[s] != 0.0f || c->iso[s] != 0.0f))
                return fail(c, ISAACB_NOT_READY, "isaacb_update: source " + std::to_string(s) + " has no memory");
        isaacb_status r = upload_lut(c, st);
        if(r != ISAACB_OK)
            return r;
        c->updateLaunches = 0;
        if(c->renderer == ISAACB_RENDERER_COMBINED)
        {
            r = compact_guarded(c, st);
            if(r != ISAACB_OK)
                return r;
            if(!c->advectedThisFrame)
            {
                r = advect_fields(c, st);
                if(r != ISAACB_OK)
                    return r;
            }
            c->advectedThisFrame = false;
            c->g.yfast = slot_order_for_camera(c);
            MergeParams p{};
            prepare_merge(c, p);
            ISAACB_CUDA(c, cudaMemsetAsync(c->emptyDev, 0, sizeof(unsigned int), st), "empty brick counter");
            {
                for(int k = 0; k < ISAACB_TIMING_SLOTS; ++k)
                    c->evUsed[k] = false;
                PhaseTimer t(c, 0, st);
                c->updateLaunches += uint32_t(launch_merge(p, st));
            }
            if(!p.writeIso && c->isoWritten)
            {
                // the reference's iso texture is all zero when no source has an iso threshold
                ISAACB_CUDA(
                    c,
                    cudaMemsetAsync(c->isoLin, 0, size_t(c->g.ls[0]) * c->g.ls[1] * c->g.ls[2] * 4, st),
                    "iso clear");
                ISAACB_CUDA(c, cudaMemsetAsync(c->isoFlag, 0, brick_count(c->g), st), "iso flag clear");
            }
            c->isoWritten = p.writeIso != 0;
        }
        else
        {
            for(int k = 0; k < c->nVol; ++k)
            {
                if(c->field[k] && (c->weight[k] != 0.0f || c->iso[k] != 0.0f))
                    return fail(c, ISAACB_INVALID_ARG, "isaacb_update: field sources are merged by the combined renderer only");
                // the reference's per-source sampler clamps a guarded persistent source's
                // coordinates to [-guard, ...] computed on an unsigned size
                // (lib/isaac/isaac_volume_kernel.hpp:206-214), which lands every sample
                // on the far corner; guarded sources take the combined renderer here
                if(c->desc.guard_size[k] != 0 && (c->weight[k] != 0.0f || c->iso[k] != 0.0f))
                    return fail(c, ISAACB_INVALID_ARG, "isaacb_update: guarded sources need the combined renderer");
            }
            for(int k = 0; k < ISAACB_TIMING_SLOTS; ++k)
                c->evUsed[k] = false;
            if(c->timing)
            {
                cudaEventRecord(c->ev[0], st);
                c->evUsed[0] = true;
            }
            for(int s = 0; s < c->nVol; ++s)
            {
                const bool enabled = c->weight[s] != 0.0f || c->iso[s] != 0.0f;
                if(!enabled)
                    continue;
                const int fdim = int(c->desc.feature_dim[s]);
                const int ncomp = c->desc.persistent[s] ? fdim : 1;
                const size_t esz = c->storage[s] == 0 ? 4 : 2;
                const size_t bytes = brick_count(c->g) * kSlotsPerBrick * 4 * ncomp * esz;
                if(c->srcBrickBytes[s] != bytes)
                {
                    cudaFree(c->srcBricks[s]);
                    c->srcBricks[s] = nullptr;
                    c->srcBrickBytes[s] = 0;
                    ISAACB_CUDA(c, cudaMalloc(&c->srcBricks[s], bytes), "per-source brick allocation");
                    c->srcBrickBytes[s] = bytes;
                }
                SourceBrickParams p{};
                p.g = c->g;
                p.src = c->src[s];
                p.fdim = fdim;
                p.ncomp = ncomp;
                p.applyChain = c->desc.persistent[s] ? 0 : 1;
                p.dtype = c->storage[s];
                p.chain = c->chain[s];
                p.out = c->srcBricks[s];
                launch_source_bricks(p, st);
                c->updateLaunches++;
            }
            if(c->timing)
                cudaEventRecord(c->ev[1], st);
        }
        ISAACB_CUDA(c, cudaGetLastError(), "isaacb_update launch");
        return ISAACB_OK;
    }

    isaacb_status isaacb_render(isaacb_ctx* c, void* stream, uint8_t* rgba_dev)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        if(!c->cameraSet)
            return fail(c, ISAACB_NOT_READY, "isaacb_render: camera not set");
        for(int s = 0; s < c->nPart; ++s)
            if(!c->partSet[s] && c->weight[c->nVol + s] != 0.0f)
                return fail(c, ISAACB_NOT_READY, "isaacb_render: particle source without memory");
        cudaStream_t st = (cudaStream_t) stream;
        isaacb_status r = upload_lut(c, st);
        if(r != ISAACB_OK)
            return r;
        FrameParams p{};
        fill_view(c, p.v);
        p.g = c->g;
        p.ts = c->ts;
        p.interpolation = c->interpolation;
        p.step = c->step;
        p.bg = make_float4(c->bg[0], c->bg[1], c->bg[2], c->bg[3]);
        p.bgSwizzled = make_float4(c->bg[3], c->bg[2], c->bg[1], 0.0f);
        p.renderMode = c->renderMode;
        p.aoWeight = c->aoWeight;
        p.aoFilter = c->aoFilter;
        p.aoSamples = c->aoSamples;
        std::memcpy(p.aoOffsets, c->aoOffsets, sizeof(p.aoOffsets));
        p.totalWeightAll = 0.0f;
        for(int s = 0; s < c->nTotal; ++s)
            p.totalWeightAll += c->weight[s];
        p.emptyCount = c->emptyDev;
        p.lut = c->lutDev;
        p.volQ = c->volQ;
        p.isoAQ = c->isoAQ;
        p.isoLin = c->isoLin;
        p.volFlag = c->volFlag;
        p.isoFlag = c->isoFlag;
        p.nVol = c->nVol;
        p.nPart = c->nPart;
        p.pscale = make_float3(
            float(c->g.lss[0]) / float(c->g.lps[0] ? c->g.lps[0] : 1),
            float(c->g.lss[1]) / float(c->g.lps[1] ? c->g.lps[1] : 1),
            float(c->g.lss[2]) / float(c->g.lps[2] ? c->g.lps[2] : 1));
        for(int s = 0; s < c->nPart; ++s)
        {
            ParticleSrc P = c->part[s];
            const int cs = c->nVol + s;
            P.fdim = int32_t(c->desc.feature_dim[cs]);
            P.weight = c->weight[cs];
            P.lutBase = cs * c->ts;
            P.chain = c->chain[cs];
            p.part[s] = P;
        }
        for(int s = 0; s < c->nVol; ++s)
        {
            PerSourceSrc& S = p.ps[s];
            S.bricks = c->srcBricks[s];
            S.dtype = c->storage[s];
            S.persistent = int32_t(c->desc.persistent[s]);
            S.fdim = int32_t(c->desc.feature_dim[s]);
            S.ncomp = S.persistent ? S.fdim : 1;
            S.weight = c->weight[s];
            S.iso = c->iso[s];
            S.chain = c->chain[s];
            if(c->renderer == ISAACB_RENDERER_PER_SOURCE && (S.weight != 0.0f || S.iso != 0.0f) && !S.bricks)
                return fail(c, ISAACB_NOT_READY, "isaacb_render: per-source bricks missing; call isaacb_update");
        }
        p.psPre = c->psPre;
        p.negZero = -0.0f;
        p.color = c->color;
        p.depth = c->depth;
        p.normal = c->normal;
        p.ao = c->ao;
        p.counters = nullptr;
        if(c->counting)
        {
            ISAACB_CUDA(c, cudaMemsetAsync(c->counters, 0, 2 * sizeof(unsigned long long), st), "counter reset");
            p.counters = c->counters;
        }
        c->renderLaunches = 0;
        for(int k = 1; k < ISAACB_TIMING_SLOTS; ++k)
            c->evUsed[k] = false;
        {
            PhaseTimer t(c, 1, st);
            launch_clear_particles(p, st);
        }
        c->renderLaunches++;
        if(c->renderer == ISAACB_RENDERER_COMBINED)
        {
            if(any_iso_active(c))
            {
                PhaseTimer t(c, 2, st);
                launch_iso(p, st);
                c->renderLaunches++;
            }
        }
        else
        {
            PhaseTimer t(c, 2, st);
            launch_iso_per_source(p, st);
            c->renderLaunches++;
        }
        if(c->aoEnabled && c->aoWeight > 0.0f)
        {
            PhaseTimer t(c, 3, st);
            launch_ssao(p, st);
            c->renderLaunches++;
        }
        {
            PhaseTimer t(c, 4, st);
            if(c->renderer == ISAACB_RENDERER_COMBINED)
            {
                launch_shade_volume(p, p.totalWeightAll > 0.0f, st);
                c->renderLaunches++;
            }
            else
                c->renderLaunches += uint32_t(launch_shade_volume_per_source(p, st));
        }
        ISAACB_CUDA(c, cudaGetLastError(), "isaacb_render launch");
        if(rgba_dev)
        {
            const size_t bytes = size_t(c->desc.framebuffer[0]) * c->desc.framebuffer[1] * 4;
            ISAACB_CUDA(c, cudaMemcpyAsync(rgba_dev, c->color, bytes, cudaMemcpyDeviceToDevice, st), "frame copy");
        }
        return ISAACB_OK;
    }

    isaacb_status isaacb_frame(isaacb_ctx* c, void* stream, uint8_t* rgba_host)
    {
        if(!c || !rgba_host)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_frame: null argument");
        isaacb_status r = isaacb_update(c, stream);
        if(r != ISAACB_OK)
            return r;
        r = isaacb_render(c, stream, nullptr);
        if(r != ISAACB_OK)
            return r;
        cudaStream_t st = (cudaStream_t) stream;
        const size_t bytes = size_t(c->desc.framebuffer[0]) * c->desc.framebuffer[1] * 4;
        ISAACB_CUDA(c, cudaMemcpyAsync(rgba_host, c->color, bytes, cudaMemcpyDeviceToHost, st), "frame readback");
        int32_t flag = 0;
        ISAACB_CUDA(c, cudaMemcpyAsync(&flag, c->errorFlag, sizeof(flag), cudaMemcpyDeviceToHost, st), "error flag");
        ISAACB_CUDA(c, cudaStreamSynchronize(st), "isaacb_frame");
        if(flag)
        {
            cudaMemsetAsync(c->errorFlag, 0, sizeof(int32_t), st);
            return fail(c, ISAACB_TIMEOUT, "isaacb_frame: a bounded device wait gave up; the frame is incomplete");
        }
        return ISAACB_OK;
    }

    isaacb_status isaacb_framebuffer(isaacb_ctx* c, uint8_t** rgba_dev)
    {
        if(!c || !rgba_dev)
            return ISAACB_INVALID_ARG;
        *rgba_dev = reinterpret_cast<uint8_t*>(c->color);
        return ISAACB_OK;
    }

    isaacb_status isaacb_minmax(isaacb_ctx* c, void* stream, float* mn, float* mx)
    {
        if(!c || !mn || !mx)
            return fail(c, ISAACB_INVALID_ARG, "isaacb_minmax: null argument");
        cudaStream_t st = (cudaStream_t) stream;
        {
            const isaacb_status r = compact_guarded(c, st);
            if(r != ISAACB_OK)
                return r;
        }
        for(int s = 0; s < c->nTotal; ++s)
        {
            MinMaxParams p{};
            p.g = c->g;
            p.chain = c->chain[s];
            p.fdim = int32_t(c->desc.feature_dim[s]);
            p.partial = c->mmPartial;
            p.keys = c->mmKeys;
            if(s < c->nVol)
            {
                if(!c->src[s])
                    return fail(c, ISAACB_NOT_READY, "isaacb_minmax: source without memory");
                p.src = source_data(c, s);
                p.particle = 0;
            }
            else
            {
                const ParticleSrc& P = c->part[s - c->nVol];
                if(!c->partSet[s - c->nVol])
                    return fail(c, ISAACB_NOT_READY, "isaacb_minmax: particle source without memory");
                p.offsets = P.offsets;
                p.attr = P.attr;
                p.particle = 1;
            }
            launch_minmax(p, minmax_blocks(p), c->mmResult, st);
            float res[2];
            ISAACB_CUDA(c, cudaMemcpyAsync(res, c->mmResult, sizeof(res), cudaMemcpyDeviceToHost, st), "minmax read");
            ISAACB_CUDA(c, cudaStreamSynchronize(st), "minmax");
            if(res[0] == 0.0f || res[1] == 0.0f)
            {
                // +0 and -0 compare equal: the reference keeps the first in its scan order
                const unsigned long long init[2] = {ULLONG_MAX, ULLONG_MAX};
                ISAACB_CUDA(c, cudaMemcpyAsync(c->mmKeys, init, sizeof(init), cudaMemcpyHostToDevice, st), "keys");
                launch_minmax_zero_keys(p, st);
                unsigned long long keys[2];
                ISAACB_CUDA(c, cudaMemcpyAsync(keys, c->mmKeys, sizeof(keys), cudaMemcpyDeviceToHost, st), "keys");
                ISAACB_CUDA(c, cudaStreamSynchronize(st), "minmax zero order");
                const float firstZero = keys[1] < keys[0] ? -0.0f : 0.0f;
                if(res[0] == 0.0f)
                    res[0] = firstZero;
                if(res[1] == 0.0f)
                    res[1] = firstZero;
            }
            mn[s] = res[0];
            mx[s] = res[1];
        }
        ISAACB_CUDA(c, cudaGetLastError(), "isaacb_minmax");
        return ISAACB_OK;
    }

    isaacb_status isaacb_get_gbuffer(isaacb_ctx* c, void* stream, float* depth, float* normal, float* ao)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        cudaStream_t st = (cudaStream_t) stream;
        const size_t npix = size_t(c->desc.framebuffer[0]) * c->desc.framebuffer[1];
        if(depth)
            ISAACB_CUDA(c, cudaMemcpyAsync(depth, c->depth, npix * 4, cudaMemcpyDeviceToHost, st), "depth");
        if(normal)
            ISAACB_CUDA(c, cudaMemcpyAsync(normal, c->normal, npix * 12, cudaMemcpyDeviceToHost, st), "normal");
        if(ao)
            ISAACB_CUDA(c, cudaMemcpyAsync(ao, c->ao, npix * 4, cudaMemcpyDeviceToHost, st), "ao");
        ISAACB_CUDA(c, cudaStreamSynchronize(st), "gbuffer");
        return ISAACB_OK;
    }

    isaacb_status isaacb_get_combined(isaacb_ctx* c, void* stream, uint8_t* volume, uint8_t* iso)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        cudaStream_t st = (cudaStream_t) stream;
        const size_t n = size_t(c->g.ls[0]) * c->g.ls[1] * c->g.ls[2];
        if(volume)
        {
            uint32_t* tmp = nullptr;
            ISAACB_CUDA(c, cudaMalloc(&tmp, n * 4), "unbrick buffer");
            launch_unbrick(c->g, c->volQ, tmp, st);
            cudaError_t e = cudaMemcpyAsync(volume, tmp, n * 4, cudaMemcpyDeviceToHost, st);
            if(e == cudaSuccess)
                e = cudaStreamSynchronize(st);
            cudaFree(tmp);
            if(e != cudaSuccess)
                return cuda_fail(c, e, "combined volume readback");
        }
        if(iso)
        {
            ISAACB_CUDA(c, cudaMemcpyAsync(iso, c->isoLin, n * 4, cudaMemcpyDeviceToHost, st), "iso readback");
            ISAACB_CUDA(c, cudaStreamSynchronize(st), "iso readback");
        }
        return ISAACB_OK;
    }

    isaacb_status isaacb_get_counters(isaacb_ctx* c, void* stream, uint64_t* vol, uint64_t* iso)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        unsigned long long h[2] = {0, 0};
        cudaStream_t st = (cudaStream_t) stream;
        ISAACB_CUDA(c, cudaMemcpyAsync(h, c->counters, sizeof(h), cudaMemcpyDeviceToHost, st), "counters");
        ISAACB_CUDA(c, cudaStreamSynchronize(st), "counters");
        if(vol)
            *vol = h[0];
        if(iso)
            *iso = h[1];
        return ISAACB_OK;
    }

    isaacb_status isaacb_set_timing(isaacb_ctx* c, int32_t on)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        if(on && !c->ev[0])
            for(auto& e : c->ev)
                ISAACB_CUDA(c, cudaEventCreate(&e), "timing events");
        c->timing = on != 0;
        return ISAACB_OK;
    }

    isaacb_status isaacb_get_timing(isaacb_ctx* c, void* stream, float* ms)
    {
        if(!c || !ms)
            return ISAACB_INVALID_ARG;
        ISAACB_CUDA(c, cudaStreamSynchronize((cudaStream_t) stream), "timing sync");
        for(int k = 0; k < ISAACB_TIMING_SLOTS; ++k)
        {
            ms[k] = 0.0f;
            if(c->timing && c->evUsed[k])
                ISAACB_CUDA(c, cudaEventElapsedTime(&ms[k], c->ev[2 * k], c->ev[2 * k + 1]), "timing read");
        }
        return ISAACB_OK;
    }

    isaacb_status isaacb_get_launch_count(isaacb_ctx* c, uint32_t* upd, uint32_t* ren)
    {
        if(!c)
            return ISAACB_INVALID_ARG;
        if(upd)
            *upd = c->updateLaunches;
        if(ren)
            *ren = c->renderLaunches;
        return ISAACB_OK;
    }
}

// ---------------------------------------------------------------------------- batched views
struct isaacb_batch
{
    std::vector<isaacb_ctx*> ctxs;
    std::vector<isaacb_view> views;
    isaacb_batch_config cfg{32, 8, 0, -1};
    BatchCtx* ctxDev = nullptr;
    BatchView* viewDev = nullptr;
    BatchCtx* ctxPinned = nullptr;
    BatchView* viewPinned = nullptr;
    cudaEvent_t tableEvent = nullptr;
    int32_t* counter = nullptr;
    unsigned long long* samples = nullptr;
    bool counting = false;
    int totalTiles = 0;
    int numSMs = 148;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    bool graphUpdate = false;
    std::vector<MergeParams> graphMerges; // merge parameters a captured graph holds
    uint32_t launches = 0; // kernels the last enqueue (direct or captured) issued
};

namespace
{
    isaacb_status batch_fail(isaacb_status st, const std::string& m)
    {
        return fail(nullptr, st, m);
    }

    // a context can join a batch when a view of it is the combined volume alone
    bool batchable(const isaacb_ctx* c, std::string& why)
    {
        if(c->renderer != ISAACB_RENDERER_COMBINED)
            why = "per-source renderer";
        else if(any_iso_active(c))
            why = "iso threshold set";
        else if(c->aoEnabled && c->aoWeight > 0.0f)
            why = "SSAO enabled";
        else if([&] {
                    for(int k = 0; k < c->nVol; ++k)
                        if(c->field[k])
                            return true;
                    return false;
                }())
            why = "advected field source";
        else
        {
            for(int s = 0; s < c->nPart; ++s)
                if(c->weight[c->nVol + s] != 0.0f)
                {
                    why = "particle source with weight";
                    return false;
                }
            return true;
        }
        return false;
    }

    void view_inverse(const double* proj, const double* mv, float* out)
    {
        float P[16], MV[16], PM[16];
        for(int i = 0; i < 16; ++i)
        {
            P[i] = float(proj[i]);
            MV[i] = float(mv[i]);
        }
        mul4(P, MV, PM);
        inverse4(PM, out);
    }

    // host mirror of the device tables from the contexts' current state; uploaded on `st`
    isaacb_status batch_refresh(isaacb_batch* b, cudaStream_t st)
    {
        if(cudaEventSynchronize(b->tableEvent) != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, "batch table staging wait");
        for(size_t i = 0; i < b->ctxs.size(); ++i)
        {
            isaacb_ctx* c = b->ctxs[i];
            BatchCtx& t = b->ctxPinned[i];
            std::memset(&t, 0, sizeof(t));
            t.g = c->g;
            t.volQ = c->volQ;
            t.volFlag = c->volFlag;
            t.step = c->step;
            t.totalWeightAll = 0.0f;
            for(int s = 0; s < c->nTotal; ++s)
                t.totalWeightAll += c->weight[s];
            t.interpolation = c->interpolation;
            t.skipEmpty = b->cfg.skip_empty >= 0 ? (b->cfg.skip_empty != 0 ? 1 : 0) : -1;
            t.emptyCount = c->emptyDev;
            t.volume = t.totalWeightAll > 0.0f ? 1 : 0;
            t.renderMode = c->renderMode;
            t.aoWeight = c->aoWeight;
            t.bg = make_float4(c->bg[0], c->bg[1], c->bg[2], c->bg[3]);
            t.bgSwizzled = make_float4(c->bg[3], c->bg[2], c->bg[1], 0.0f);
            t.scale = make_float3(c->desc.scale[0], c->desc.scale[1], c->desc.scale[2]);
            t.clipCount = c->clipCount;
            std::memcpy(t.clipPos, c->clipPos, sizeof(t.clipPos));
            std::memcpy(t.clipNrm, c->clipNrm, sizeof(t.clipNrm));
        }
        int base = 0;
        for(size_t v = 0; v < b->views.size(); ++v)
        {
            const isaacb_view& iv = b->views[v];
            BatchView& t = b->viewPinned[v];
            view_inverse(iv.projection, iv.modelview, t.inv);
            t.W = int32_t(iv.width);
            t.H = int32_t(iv.height);
            t.ctx = int32_t(iv.ctx_index);
            t.tilesX = int32_t((iv.width + b->cfg.tile_w - 1) / b->cfg.tile_w);
            t.tiles = t.tilesX * int32_t((iv.height + b->cfg.tile_h - 1) / b->cfg.tile_h);
            t.tileBase = base;
            t.out = reinterpret_cast<uchar4*>(iv.rgba_dev);
            base += t.tiles;
        }
        b->totalTiles = base;
        cudaError_t e = cudaMemcpyAsync(b->ctxDev, b->ctxPinned, b->ctxs.size() * sizeof(BatchCtx), cudaMemcpyHostToDevice, st);
        if(e == cudaSuccess)
            e = cudaMemcpyAsync(b->viewDev, b->viewPinned, b->views.size() * sizeof(BatchView), cudaMemcpyHostToDevice, st);
        if(e == cudaSuccess)
            e = cudaEventRecord(b->tableEvent, st);
        if(e != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, std::string("batch table upload: ") + cudaGetErrorString(e));
        return ISAACB_OK;
    }

    int batch_blocks(const isaacb_batch* b)
    {
        const int maxb = batch_max_blocks_per_sm();
        const int per = (b->cfg.blocks_per_sm == 0 || int(b->cfg.blocks_per_sm) > maxb) ? maxb : int(b->cfg.blocks_per_sm);
        return b->numSMs * per;
    }

    // the stream work of one batch frame; `capture` leaves out the read-back of the empty-brick counts
    isaacb_status batch_enqueue(isaacb_batch* b, cudaStream_t st, bool update, bool capture)
    {
        b->launches = 0;
        if(update)
        {
            for(isaacb_ctx* c : b->ctxs)
            {
                for(int s = 0; s < c->nVol; ++s)
                    if(!c->src[s] && (c->weight[s] != 0.0f || c->iso[s] != 0.0f))
                        return batch_fail(ISAACB_NOT_READY, "isaacb_batch: a source has no memory");
                if(compact_guarded(c, st) != ISAACB_OK)
                    return batch_fail(ISAACB_CUDA_ERROR, std::string("isaacb_batch: ") + c->lastError);
                // the batch kernel's views look from every side: x-fastest slots
                c->g.yfast = 0;
                MergeParams p{};
                prepare_merge(c, p);
                if(capture)
                    b->graphMerges.push_back(p);
                if(cudaMemsetAsync(c->emptyDev, 0, sizeof(unsigned int), st) != cudaSuccess)
                    return batch_fail(ISAACB_CUDA_ERROR, "isaacb_batch: empty brick counter");
                b->launches += uint32_t(launch_merge(p, st));
            }
        }
        if(cudaMemsetAsync(b->counter, 0, sizeof(int32_t), st) != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, "isaacb_batch: queue reset");
        BatchParams bp{};
        bp.ctxs = b->ctxDev;
        bp.views = b->viewDev;
        bp.nViews = int32_t(b->views.size());
        bp.totalTiles = b->totalTiles;
        bp.tileW = int32_t(b->cfg.tile_w);
        bp.tileH = int32_t(b->cfg.tile_h);
        bp.counter = b->counter;
        bp.samples = b->counting ? b->samples : nullptr;
        if(b->counting && cudaMemsetAsync(b->samples, 0, sizeof(unsigned long long), st) != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, "isaacb_batch: sample counter reset");
        launch_batch(bp, batch_blocks(b), st);
        b->launches++;
        const cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, std::string("isaacb_batch launch: ") + cudaGetErrorString(e));
        return ISAACB_OK;
    }

    isaacb_status batch_upload_luts(isaacb_batch* b, cudaStream_t st)
    {
        for(isaacb_ctx* c : b->ctxs)
        {
            const isaacb_status r = upload_lut(c, st);
            if(r != ISAACB_OK)
                return batch_fail(r, c->lastError);
        }
        return ISAACB_OK;
    }

    void batch_drop_graph(isaacb_batch* b)
    {
        if(b->graphExec)
            cudaGraphExecDestroy(b->graphExec);
        if(b->graph)
            cudaGraphDestroy(b->graph);
        b->graphExec = nullptr;
        b->graph = nullptr;
        b->graphMerges.clear();
    }

    // true when a context's merge parameters changed since the graph was captured
    bool batch_graph_stale(const isaacb_batch* b)
    {
        if(!b->graphUpdate)
            return false;
        for(size_t i = 0; i < b->ctxs.size(); ++i)
        {
            MergeParams p{};
            prepare_merge(b->ctxs[i], p);
            if(i >= b->graphMerges.size() || std::memcmp(&p, &b->graphMerges[i], sizeof(MergeParams)) != 0)
                return true;
        }
        return false;
    }
} // namespace

extern "C"
{
    isaacb_status isaacb_batch_create(
        isaacb_ctx* const* ctxs,
        uint32_t n_ctx,
        const isaacb_view* views,
        uint32_t n_views,
        isaacb_batch** out)
    {
        if(!ctxs || !views || !out || n_ctx == 0 || n_views == 0 || n_ctx > 4096 || n_views > 4096)
            return batch_fail(ISAACB_INVALID_ARG, "isaacb_batch_create: bad arguments");
        *out = nullptr;
        for(uint32_t i = 0; i < n_ctx; ++i)
        {
            std::string why;
            if(!ctxs[i])
                return batch_fail(ISAACB_INVALID_ARG, "isaacb_batch_create: null context");
            if(!batchable(ctxs[i], why))
                return batch_fail(ISAACB_INVALID_ARG, "isaacb_batch_create: context " + std::to_string(i) + ": " + why);
        }
        for(uint32_t v = 0; v < n_views; ++v)
            if(views[v].ctx_index >= n_ctx || views[v].width == 0 || views[v].height == 0 || views[v].width > 16384
               || views[v].height > 16384 || !views[v].rgba_dev)
                return batch_fail(ISAACB_INVALID_ARG, "isaacb_batch_create: bad view " + std::to_string(v));
        isaacb_batch* b = new isaacb_batch;
        b->ctxs.assign(ctxs, ctxs + n_ctx);
        b->views.assign(views, views + n_views);
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, dev);
        cudaError_t e = cudaMalloc(&b->ctxDev, n_ctx * sizeof(BatchCtx));
        if(e == cudaSuccess)
            e = cudaMalloc(&b->viewDev, n_views * sizeof(BatchView));
        if(e == cudaSuccess)
            e = cudaMallocHost(&b->ctxPinned, n_ctx * sizeof(BatchCtx));
        if(e == cudaSuccess)
            e = cudaMallocHost(&b->viewPinned, n_views * sizeof(BatchView));
        if(e == cudaSuccess)
            e = cudaMalloc(&b->counter, sizeof(int32_t));
        if(e == cudaSuccess)
            e = cudaMalloc(&b->samples, sizeof(unsigned long long));
        if(e == cudaSuccess)
            e = cudaEventCreateWithFlags(&b->tableEvent, cudaEventDisableTiming);
        if(e != cudaSuccess)
        {
            isaacb_batch_destroy(b);
            return batch_fail(e == cudaErrorMemoryAllocation ? ISAACB_OOM : ISAACB_CUDA_ERROR, "isaacb_batch_create: allocation");
        }
        *out = b;
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_destroy(isaacb_batch* b)
    {
        if(!b)
            return ISAACB_OK;
        batch_drop_graph(b);
        cudaFree(b->ctxDev);
        cudaFree(b->viewDev);
        if(b->ctxPinned)
            cudaFreeHost(b->ctxPinned);
        if(b->viewPinned)
            cudaFreeHost(b->viewPinned);
        cudaFree(b->counter);
        cudaFree(b->samples);
        if(b->tableEvent)
            cudaEventDestroy(b->tableEvent);
        delete b;
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_set_config(isaacb_batch* b, const isaacb_batch_config* cfg)
    {
        if(!b || !cfg || cfg->tile_w * cfg->tile_h != 256 || cfg->tile_w % 8 != 0 || cfg->tile_h % 4 != 0
           || cfg->skip_empty < -1 || cfg->skip_empty > 1)
            return batch_fail(ISAACB_INVALID_ARG, "isaacb_batch_set_config: tiles must be 256 pixels, width % 8, height % 4");
        b->cfg = *cfg;
        batch_drop_graph(b);
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_get_config(const isaacb_batch* b, isaacb_batch_config* cfg)
    {
        if(!b || !cfg)
            return ISAACB_INVALID_ARG;
        *cfg = b->cfg;
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_set_camera(isaacb_batch* b, uint32_t v, const double* proj, const double* mv)
    {
        if(!b || v >= b->views.size() || !proj || !mv)
            return batch_fail(ISAACB_INVALID_ARG, "isaacb_batch_set_camera: bad arguments");
        std::memcpy(b->views[v].projection, proj, sizeof(double) * 16);
        std::memcpy(b->views[v].modelview, mv, sizeof(double) * 16);
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_render(isaacb_batch* b, void* stream, int32_t update)
    {
        if(!b)
            return ISAACB_INVALID_ARG;
        cudaStream_t st = (cudaStream_t) stream;
        isaacb_status r = batch_upload_luts(b, st);
        if(r == ISAACB_OK)
            r = batch_refresh(b, st);
        if(r == ISAACB_OK)
            r = batch_enqueue(b, st, update != 0, false);
        return r;
    }

    isaacb_status isaacb_batch_capture(isaacb_batch* b, void* stream, int32_t update)
    {
        if(!b || !stream)
            return batch_fail(ISAACB_INVALID_ARG, "isaacb_batch_capture: needs a non-default stream");
        cudaStream_t st = (cudaStream_t) stream;
        isaacb_status r = batch_upload_luts(b, st);
        if(r == ISAACB_OK)
            r = batch_refresh(b, st);
        if(r != ISAACB_OK)
            return r;
        batch_drop_graph(b);
        if(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, "isaacb_batch_capture: begin capture");
        r = batch_enqueue(b, st, update != 0, true);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(st, &g);
        if(r != ISAACB_OK || e != cudaSuccess)
        {
            if(g)
                cudaGraphDestroy(g);
            return r != ISAACB_OK ? r : batch_fail(ISAACB_CUDA_ERROR, "isaacb_batch_capture: end capture");
        }
        if(cudaGraphInstantiate(&b->graphExec, g, 0) != cudaSuccess)
        {
            cudaGraphDestroy(g);
            return batch_fail(ISAACB_CUDA_ERROR, "isaacb_batch_capture: instantiate");
        }
        b->graph = g;
        b->graphUpdate = update != 0;
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_launch_graph(isaacb_batch* b, void* stream)
    {
        if(!b || !b->graphExec)
            return batch_fail(ISAACB_NOT_READY, "isaacb_batch_launch_graph: no captured graph");
        cudaStream_t st = (cudaStream_t) stream;
        // functors, weights, storage or source memory changed: the merges in the graph are out of date
        if(batch_graph_stale(b))
        {
            const bool update = b->graphUpdate;
            const isaacb_status rc = isaacb_batch_capture(b, stream, update ? 1 : 0);
            if(rc != ISAACB_OK)
                return rc;
        }
        // cameras and frame settings live in device tables the graph reads
        isaacb_status r = batch_upload_luts(b, st);
        if(r == ISAACB_OK)
            r = batch_refresh(b, st);
        if(r != ISAACB_OK)
            return r;
        const cudaError_t e = cudaGraphLaunch(b->graphExec, st);
        if(e != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, std::string("isaacb_batch_launch_graph: ") + cudaGetErrorString(e));
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_autotune(isaacb_batch* b, void* stream, isaacb_batch_config* best, float* best_ms)
    {
        if(!b)
            return ISAACB_INVALID_ARG;
        cudaStream_t st = (cudaStream_t) stream;
        const uint32_t shapes[4][2] = {{32, 8}, {16, 16}, {8, 32}, {64, 4}};
        const int maxb = batch_max_blocks_per_sm();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        isaacb_batch_config keep = b->cfg, bestCfg = b->cfg;
        float bestT = 3.0e38f;
        isaacb_status r = ISAACB_OK;
        for(const auto& sh : shapes)
            for(int per = 1; per <= maxb && r == ISAACB_OK; per = (per == maxb ? maxb + 1 : std::min(maxb, per * 2)))
                for(int skip = 0; skip <= 1 && r == ISAACB_OK; ++skip)
                {
                    b->cfg = isaacb_batch_config{sh[0], sh[1], uint32_t(per), skip};
                    r = isaacb_batch_render(b, st, 0); // warm-up
                    cudaEventRecord(e0, st);
                    for(int k = 0; k < 3 && r == ISAACB_OK; ++k)
                        r = isaacb_batch_render(b, st, 0);
                    cudaEventRecord(e1, st);
                    cudaEventSynchronize(e1);
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, e0, e1);
                    ms /= 3.0f;
                    if(r == ISAACB_OK && ms < bestT)
                    {
                        bestT = ms;
                        bestCfg = b->cfg;
                    }
                }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        b->cfg = r == ISAACB_OK ? bestCfg : keep;
        batch_drop_graph(b);
        if(best)
            *best = b->cfg;
        if(best_ms)
            *best_ms = bestT;
        return r;
    }

    isaacb_status isaacb_batch_set_counting(isaacb_batch* b, int32_t on)
    {
        if(!b)
            return ISAACB_INVALID_ARG;
        b->counting = on != 0;
        batch_drop_graph(b);
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_get_launch_count(isaacb_batch* b, uint32_t* launches)
    {
        if(!b || !launches)
            return ISAACB_INVALID_ARG;
        *launches = b->launches;
        return ISAACB_OK;
    }

    isaacb_status isaacb_batch_get_samples(isaacb_batch* b, void* stream, uint64_t* samples)
    {
        if(!b || !samples)
            return ISAACB_INVALID_ARG;
        unsigned long long h = 0;
        cudaStream_t st = (cudaStream_t) stream;
        if(cudaMemcpyAsync(&h, b->samples, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess
           || cudaStreamSynchronize(st) != cudaSuccess)
            return batch_fail(ISAACB_CUDA_ERROR, "isaacb_batch_get_samples");
        *samples = h;
        return ISAACB_OK;
    }
}
