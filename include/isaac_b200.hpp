/* isaac_b200.hpp -- header-only C++ front end with the roles of ISAAC's
 * IsaacVisualization template (lib/isaac.hpp:58-3036) over the C ABI of
 * isaac_b200.h.  Compile the including translation unit with nvcc: the front
 * end instantiates, per user source type, a gather kernel that calls the
 * user's device operator[] (volume sources) or getIterator(cell) (particle
 * sources), exactly the interfaces the reference reads
 * (example/example.cpp:36-228).  Everything else goes through the C ABI.
 *
 * Differences from the reference class:
 *  - no alpaka host/accelerator/stream objects, no server URL/port, no MPI;
 *    an optional cudaStream_t replaces the alpaka stream;
 *  - field sources (FieldSourceList, float3 vector fields that are advected) become
 *    the last volume sources of the context, after every plain volume source, and
 *    are flagged with isaacb_set_field_source -- the merge order of the reference;
 *    advection runs with the combined renderer;
 *  - glm vector types are replaced by isaacb::float_dim<N> and isaacb::int3v,
 *    which have the same component names (x, y, z, w) and operator[];
 *  - a volume source may expose `const float* linearData() const` (x-fastest,
 *    featureDim floats per voxel, guardSize cells on every side); then its memory
 *    is read in place instead of gathered through operator[] every frame.  A
 *    gathered source is copied without its guard cells.
 */
#ifndef ISAAC_B200_HPP
#define ISAAC_B200_HPP

#include "isaac_b200.h"

#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include <cuda_runtime.h>

namespace isaacb
{
    // ---------------------------------------------------------------- small vector types
    template<int N>
    struct float_dim;
    template<>
    struct float_dim<1>
    {
        float x;
        __host__ __device__ float& operator[](int) { return x; }
        __host__ __device__ float operator[](int) const { return x; }
    };
    template<>
    struct float_dim<2>
    {
        float x, y;
        __host__ __device__ float& operator[](int i) { return i == 0 ? x : y; }
        __host__ __device__ float operator[](int i) const { return i == 0 ? x : y; }
    };
    template<>
    struct float_dim<3>
    {
        float x, y, z;
        __host__ __device__ float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
        __host__ __device__ float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    };
    template<>
    struct float_dim<4>
    {
        float x, y, z, w;
        __host__ __device__ float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
        __host__ __device__ float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
    };
    struct int3v
    {
        int x, y, z;
    };
    struct uint3v
    {
        unsigned x, y, z;
    };

    class Error : public std::runtime_error
    {
    public:
        Error(isaacb_status s, const std::string& m) : std::runtime_error(m), status(s) {}
        isaacb_status status;
    };

    namespace detail
    {
        inline void check(isaacb_status s, const isaacb_ctx* ctx, const char* what)
        {
            if(s != ISAACB_OK)
                throw Error(s, std::string(what) + ": " + isaacb_last_error(ctx));
        }
        inline void cuda(cudaError_t e, const char* what)
        {
            if(e != cudaSuccess)
                throw Error(ISAACB_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
        }

        template<class T, class = void>
        struct has_linear_data : std::false_type
        {
        };
        template<class T>
        struct has_linear_data<T, std::void_t<decltype(std::declval<const T&>().linearData())>> : std::true_type
        {
        };

        // gather of a volume source through its operator[] into x-fastest floats
        template<class Source>
        __global__ void gather_volume(const Source src, float* out, int X, int Y, int Z)
        {
            const size_t n = size_t(X) * Y * Z;
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                const int x = int(i % X), y = int((i / X) % Y), z = int(i / (size_t(X) * Y));
                const auto v = src[int3v{x, y, z}];
                for(int c = 0; c < int(Source::featureDim); ++c)
                    out[i * Source::featureDim + c] = v[c];
            }
        }

        // particle cell list: counts, then positions / attributes / radii at the scanned offsets
        template<class Source>
        __global__ void count_particles(const Source src, uint32_t* counts, int PX, int PY, int PZ)
        {
            const size_t n = size_t(PX) * PY * PZ;
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                const uint3v c{unsigned(i % PX), unsigned((i / PX) % PY), unsigned(i / (size_t(PX) * PY))};
                counts[i] = uint32_t(src.getIterator(c).size);
            }
        }
        template<class Source>
        __global__ void fill_particles(
            const Source src,
            const uint32_t* offsets,
            float* pos,
            float* attr,
            float* radius,
            int PX,
            int PY,
            int PZ)
        {
            const size_t n = size_t(PX) * PY * PZ;
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                const uint3v c{unsigned(i % PX), unsigned((i / PX) % PY), unsigned(i / (size_t(PX) * PY))};
                auto it = src.getIterator(c);
                uint32_t k = offsets[i];
                for(size_t j = 0; j < size_t(it.size); ++j, ++k)
                {
                    const auto p = it.getPosition();
                    pos[3 * size_t(k)] = p.x;
                    pos[3 * size_t(k) + 1] = p.y;
                    pos[3 * size_t(k) + 2] = p.z;
                    const auto a = it.getAttribute();
                    for(int d = 0; d < int(Source::featureDim); ++d)
                        attr[size_t(k) * Source::featureDim + d] = a[d];
                    radius[k] = it.getRadius();
                    it.next();
                }
            }
        }
        // single-block exclusive scan of the cell counts (n+1 offsets); a template so that
        // every translation unit including this header may instantiate it
        template<int Unused = 0>
        __global__ void exclusive_scan(const uint32_t* counts, uint32_t* offsets, size_t n)
        {
            __shared__ uint32_t part[1024];
            const size_t chunk = (n + 1023) / 1024;
            const size_t b = threadIdx.x * chunk, e = b + chunk < n ? b + chunk : n;
            uint32_t s = 0;
            for(size_t i = b; i < e; ++i)
                s += counts[i];
            part[threadIdx.x] = s;
            __syncthreads();
            if(threadIdx.x == 0)
            {
                uint32_t acc = 0;
                for(int t = 0; t < 1024; ++t)
                {
                    const uint32_t v = part[t];
                    part[t] = acc;
                    acc += v;
                }
                offsets[n] = acc;
            }
            __syncthreads();
            uint32_t acc = part[threadIdx.x];
            for(size_t i = b; i < e; ++i)
            {
                offsets[i] = acc;
                acc += counts[i];
            }
        }

        template<class Tuple, class F, std::size_t... I>
        void for_each_impl(Tuple& t, F&& f, std::index_sequence<I...>)
        {
            (f(std::integral_constant<std::size_t, I>{}, std::get<I>(t)), ...);
        }
        template<class Tuple, class F>
        void for_each(Tuple& t, F&& f)
        {
            for_each_impl(t, std::forward<F>(f), std::make_index_sequence<std::tuple_size<Tuple>::value>{});
        }
    } // namespace detail

    // DefaultController (lib/isaac/isaac_controllers.hpp:23-43): glm::perspective(45.0, w/h,
    // 0.002, 100) with 45.0 read as radians, column major
    struct DefaultController
    {
        static std::array<double, 16> projection(uint32_t w, uint32_t h)
        {
            const double fovy = 45.0, aspect = double(w) / double(h), zn = 0.002, zf = 100.0;
            const double t = std::tan(fovy / 2.0);
            std::array<double, 16> m{};
            m[0] = 1.0 / (aspect * t);
            m[5] = 1.0 / t;
            m[10] = -(zf + zn) / (zf - zn);
            m[11] = -1.0;
            m[14] = -(2.0 * zf * zn) / (zf - zn);
            return m;
        }
    };

    template<class... S>
    using SourceList = std::tuple<S...>;

    template<
        class VolumeSourceList,
        class FieldSourceList,
        class ParticleList,
        int TransferSize = 1024,
        class Controller = DefaultController>
    class IsaacVisualization
    {
        static constexpr int nPlain = int(std::tuple_size<VolumeSourceList>::value);
        static constexpr int nField = int(std::tuple_size<FieldSourceList>::value);
        static constexpr int nVol = nPlain + nField; // field sources follow the plain ones
        static constexpr int nPart = int(std::tuple_size<ParticleList>::value);
        static constexpr int nTotal = nVol + nPart;

    public:
        struct Function
        {
            std::string source;
            int32_t errorCode = 0;
        };

        IsaacVisualization(
            const std::string& name,
            std::array<uint32_t, 2> framebufferSize,
            std::array<uint32_t, 3> globalSize,
            std::array<uint32_t, 3> localSize,
            std::array<uint32_t, 3> localParticleSize,
            std::array<int32_t, 3> position,
            VolumeSourceList& volumeSources,
            FieldSourceList& fieldSources,
            ParticleList& particleSources,
            std::array<float, 3> scale = {1.0f, 1.0f, 1.0f},
            cudaStream_t stream = nullptr)
            : name_(name)
            , fb_(framebufferSize)
            , local_(localSize)
            , localParticle_(localParticleSize)
            , volumeSources_(volumeSources)
            , fieldSources_(fieldSources)
            , particleSources_(particleSources)
            , stream_(stream)
        {
            isaacb_desc d{};
            d.framebuffer[0] = fb_[0];
            d.framebuffer[1] = fb_[1];
            for(int i = 0; i < 3; ++i)
            {
                d.global_size[i] = globalSize[i];
                d.local_size[i] = localSize[i];
                d.local_particle_size[i] = localParticleSize[i];
                d.position[i] = position[i];
                d.scale[i] = scale[i];
            }
            d.transfer_size = TransferSize;
            d.n_volume_sources = nVol;
            d.n_particle_sources = nPart;
            detail::for_each(volumeSources_, [&](auto I, auto& s) {
                using S = std::decay_t<decltype(s)>;
                d.feature_dim[I] = uint32_t(S::featureDim);
                d.persistent[I] = S::persistent ? 1u : 0u;
                // memory read in place keeps its guard cells; a gathered copy is the interior
                d.guard_size[I] = detail::has_linear_data<S>::value ? uint32_t(S::guardSize) : 0u;
            });
            detail::for_each(fieldSources_, [&](auto I, auto& s) {
                using S = std::decay_t<decltype(s)>;
                static_assert(S::featureDim == 3, "a field source is a float3 vector field");
                d.feature_dim[nPlain + I] = 3u;
                d.persistent[nPlain + I] = S::persistent ? 1u : 0u;
                d.guard_size[nPlain + I] = detail::has_linear_data<S>::value ? uint32_t(S::guardSize) : 0u;
            });
            detail::for_each(particleSources_, [&](auto I, auto& s) {
                using S = std::decay_t<decltype(s)>;
                d.feature_dim[nVol + I] = uint32_t(S::featureDim);
                d.persistent[nVol + I] = 1u;
            });
            detail::check(isaacb_create(&d, &ctx_), nullptr, "isaacb_create");
            for(int i = nPlain; i < nVol; ++i)
                detail::check(isaacb_set_field_source(ctx_, uint32_t(i), 1), ctx_, "field source");
            for(int i = 0; i < nTotal; ++i)
                functions[i].source = "idem";
            staging_.fill(nullptr);
            partBuf_.fill(PartBuffers{});
            projection = Controller::projection(fb_[0], fb_[1]);
            updateModelview();
            frame_.resize(size_t(fb_[0]) * fb_[1] * 4);
        }

        ~IsaacVisualization()
        {
            for(float* p : staging_)
                if(p)
                    cudaFree(p);
            for(auto& b : partBuf_)
                b.release();
            isaacb_destroy(ctx_);
        }
        IsaacVisualization(const IsaacVisualization&) = delete;
        IsaacVisualization& operator=(const IsaacVisualization&) = delete;

        // ---- steering (reference setters and JSON keys)
        std::array<Function, nTotal> functions;

        std::array<int32_t, nTotal> updateFunctions()
        {
            std::array<int32_t, nTotal> codes{};
            for(int i = 0; i < nTotal; ++i)
            {
                int32_t err = 0;
                const isaacb_status s = isaacb_set_functions(ctx_, i, functions[i].source.c_str(), &err);
                if(s != ISAACB_OK && s != ISAACB_PARSE_ERROR)
                    detail::check(s, ctx_, "updateFunctions");
                functions[i].errorCode = codes[i] = err;
            }
            return codes;
        }
        // control points of one source ("transfer points"), then updateTransfer()
        std::array<std::map<uint32_t, std::array<float, 4>>, nTotal> transferPoints;
        void updateTransfer()
        {
            for(int i = 0; i < nTotal; ++i)
            {
                if(transferPoints[i].empty())
                    continue;
                std::vector<uint32_t> keys;
                std::vector<float> rgba;
                for(auto& kv : transferPoints[i])
                {
                    keys.push_back(kv.first);
                    rgba.insert(rgba.end(), kv.second.begin(), kv.second.end());
                }
                detail::check(
                    isaacb_set_transfer(ctx_, i, uint32_t(keys.size()), keys.data(), rgba.data()),
                    ctx_,
                    "updateTransfer");
            }
        }
        void setWeight(int src, float w) { detail::check(isaacb_set_weight(ctx_, src, w), ctx_, "weight"); }
        void setIsoThreshold(int src, float v) { detail::check(isaacb_set_iso_threshold(ctx_, src, v), ctx_, "iso threshold"); }
        void setStep(float s) { detail::check(isaacb_set_step(ctx_, s), ctx_, "step"); }
        void setInterpolation(bool on) { detail::check(isaacb_set_interpolation(ctx_, on), ctx_, "interpolation"); }
        void setRenderOptimization(bool on)
        {
            detail::check(
                isaacb_set_renderer(ctx_, on ? ISAACB_RENDERER_COMBINED : ISAACB_RENDERER_PER_SOURCE),
                ctx_,
                "render optimization");
        }
        void setAmbientOcclusion(bool enabled, float weight) { detail::check(isaacb_set_ao(ctx_, enabled, weight, 0), ctx_, "ao"); }
        // "advection step", "advection weight", "advection seeding period", "advection
        // seeding duration", "seed points" (lib/isaac.hpp:1636-1662)
        void setAdvection(float stepFactor, float historyWeight, int seedingPeriod, int seedingDuration, int seedPoints)
        {
            detail::check(
                isaacb_set_advection(ctx_, stepFactor, historyWeight, seedingPeriod, seedingDuration, seedPoints),
                ctx_,
                "advection");
        }
        void setRenderMode(int m) { detail::check(isaacb_set_render_mode(ctx_, m), ctx_, "render mode"); }
        void setDitherMode(int m) { detail::check(isaacb_set_dither_mode(ctx_, m), ctx_, "dither mode"); }
        void setBackgroundColor(std::array<float, 4> rgba)
        {
            detail::check(isaacb_set_background(ctx_, rgba.data()), ctx_, "background color");
        }
        bool editClipping(uint32_t nr, float px, float py, float pz, float nx, float ny, float nz)
        {
            const float p[3] = {px, py, pz}, n[3] = {nx, ny, nz};
            return isaacb_edit_clipping(ctx_, nr, p, n) == ISAACB_OK;
        }
        void addClipping(float px, float py, float pz, float nx, float ny, float nz)
        {
            const float p[3] = {px, py, pz}, n[3] = {nx, ny, nz};
            isaacb_add_clipping(ctx_, p, n);
        }
        void removeClipping(uint32_t nr) { isaacb_remove_clipping(ctx_, nr); }

        // camera: projection from the controller, modelview = distance * rotation * translate(lookAt)
        // (updateModelview, lib/isaac.hpp:2878-2889); all column major
        std::array<double, 16> projection{};
        std::array<double, 3> lookAt{0.0, 0.0, 0.0};
        std::array<double, 9> rotation{1, 0, 0, 0, 1, 0, 0, 0, 1};
        double distance = -4.5;
        std::array<double, 16> modelview{};
        void updateModelview()
        {
            std::array<double, 16> T{}, R{}, D{};
            for(int i = 0; i < 4; ++i)
                T[i * 5] = R[i * 5] = D[i * 5] = 1.0;
            T[12] = lookAt[0];
            T[13] = lookAt[1];
            T[14] = lookAt[2];
            for(int c = 0; c < 3; ++c)
                for(int r = 0; r < 3; ++r)
                    R[c * 4 + r] = rotation[c * 3 + r];
            D[14] = distance;
            modelview = mul(mul(D, R), T);
        }
        void setCamera(const std::array<double, 16>& P, const std::array<double, 16>& MV)
        {
            projection = P;
            modelview = MV;
        }

        // ---- per frame: doVisualization (lib/isaac.hpp:1298-2104); returns the RGBA8 frame
        const uint8_t* doVisualization(void* pointer = nullptr, bool redraw = true)
        {
            prepare(pointer);
            if(!redraw)
                return frame_.data();
            detail::check(isaacb_frame(ctx_, stream_, frame_.data()), ctx_, "doVisualization");
            return frame_.data();
        }
        // min/max of every source after its functor chain ("minmax" request)
        std::pair<std::array<float, nTotal>, std::array<float, nTotal>> minMax()
        {
            prepare(nullptr);
            std::pair<std::array<float, nTotal>, std::array<float, nTotal>> r;
            detail::check(isaacb_minmax(ctx_, stream_, r.first.data(), r.second.data()), ctx_, "minMax");
            return r;
        }
        const std::vector<uint8_t>& frame() const { return frame_; }
        isaacb_ctx* context() { return ctx_; }

    private:
        struct PartBuffers
        {
            uint32_t* counts = nullptr;
            uint32_t* offsets = nullptr;
            float* pos = nullptr;
            float* attr = nullptr;
            float* radius = nullptr;
            size_t capacity = 0;
            void release()
            {
                cudaFree(counts);
                cudaFree(offsets);
                cudaFree(pos);
                cudaFree(attr);
                cudaFree(radius);
                *this = PartBuffers{};
            }
        };

        static std::array<double, 16> mul(const std::array<double, 16>& A, const std::array<double, 16>& B)
        {
            std::array<double, 16> R{};
            for(int c = 0; c < 4; ++c)
                for(int r = 0; r < 4; ++r)
                {
                    double s = 0;
                    for(int k = 0; k < 4; ++k)
                        s += A[k * 4 + r] * B[c * 4 + k];
                    R[c * 4 + r] = s;
                }
            return R;
        }

        // source update hooks (lib/isaac.hpp:249-290), gathers, particle lists, camera
        void prepare(void* pointer)
        {
            detail::for_each(volumeSources_, [&](auto I, auto& s) { prepareVolume(int(I), s, pointer); });
            detail::for_each(fieldSources_, [&](auto I, auto& s) { prepareVolume(nPlain + int(I), s, pointer); });
            detail::for_each(particleSources_, [&](auto I, auto& s) {
                using S = std::decay_t<decltype(s)>;
                s.update(true, pointer);
                gatherParticles<S>(I, s);
            });
            detail::check(isaacb_set_camera(ctx_, projection.data(), modelview.data()), ctx_, "camera");
        }

        // the source's update hook, then its memory in place (linearData) or gathered
        // through its device operator[] into a staging buffer
        template<class S>
        void prepareVolume(int I, S& s, void* pointer)
        {
            s.update(true, pointer);
            if constexpr(detail::has_linear_data<S>::value)
            {
                detail::check(isaacb_set_source(ctx_, uint32_t(I), s.linearData()), ctx_, "set source");
            }
            else
            {
                const size_t nvox = size_t(local_[0]) * local_[1] * local_[2];
                if(!staging_[I])
                    detail::cuda(cudaMalloc(&staging_[I], nvox * S::featureDim * sizeof(float)), "staging allocation");
                detail::gather_volume<S>
                    <<<148 * 8, 256, 0, stream_>>>(s, staging_[I], int(local_[0]), int(local_[1]), int(local_[2]));
                detail::cuda(cudaGetLastError(), "gather launch");
                detail::check(isaacb_set_source(ctx_, uint32_t(I), staging_[I]), ctx_, "set source");
            }
        }

        template<class S>
        void gatherParticles(int I, const S& s)
        {
            PartBuffers& b = partBuf_[I];
            const int PX = int(localParticle_[0]), PY = int(localParticle_[1]), PZ = int(localParticle_[2]);
            const size_t ncell = size_t(PX) * PY * PZ;
            if(!b.counts)
            {
                detail::cuda(cudaMalloc(&b.counts, ncell * sizeof(uint32_t)), "particle counts");
                detail::cuda(cudaMalloc(&b.offsets, (ncell + 1) * sizeof(uint32_t)), "particle offsets");
            }
            detail::count_particles<S><<<148 * 8, 256, 0, stream_>>>(s, b.counts, PX, PY, PZ);
            detail::exclusive_scan<><<<1, 1024, 0, stream_>>>(b.counts, b.offsets, ncell);
            uint32_t total = 0;
            detail::cuda(
                cudaMemcpyAsync(&total, b.offsets + ncell, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream_),
                "particle total");
            detail::cuda(cudaStreamSynchronize(stream_), "particle total");
            if(total > b.capacity)
            {
                cudaFree(b.pos);
                cudaFree(b.attr);
                cudaFree(b.radius);
                const size_t cap = total + total / 4 + 1;
                detail::cuda(cudaMalloc(&b.pos, cap * 3 * sizeof(float)), "particle positions");
                detail::cuda(cudaMalloc(&b.attr, cap * S::featureDim * sizeof(float)), "particle attributes");
                detail::cuda(cudaMalloc(&b.radius, cap * sizeof(float)), "particle radii");
                b.capacity = cap;
            }
            detail::fill_particles<S><<<148 * 8, 256, 0, stream_>>>(s, b.offsets, b.pos, b.attr, b.radius, PX, PY, PZ);
            detail::cuda(cudaGetLastError(), "particle gather");
            detail::check(
                isaacb_set_particles(ctx_, nVol + I, b.offsets, b.pos, b.attr, b.radius, 0.0f),
                ctx_,
                "set particles");
        }

        std::string name_;
        std::array<uint32_t, 2> fb_;
        std::array<uint32_t, 3> local_, localParticle_;
        VolumeSourceList& volumeSources_;
        FieldSourceList& fieldSources_;
        ParticleList& particleSources_;
        cudaStream_t stream_;
        isaacb_ctx* ctx_ = nullptr;
        std::array<float*, (nVol > 0 ? nVol : 1)> staging_;
        std::array<PartBuffers, (nPart > 0 ? nPart : 1)> partBuf_;
        std::vector<uint8_t> frame_;
    };
} // namespace isaacb

#endif /* ISAAC_B200_HPP */
