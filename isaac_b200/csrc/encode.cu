// Frame output path of the communicator (IsaacCommunicator::serverSendFrame,
// lib/isaac/isaac_communicator.hpp:214-290): the RGBA8 frame as a JPEG or as its raw
// bytes, base64-encoded, wrapped in the payload message
//   {"payload": "data:image/jpeg;base64,<text>"}   (raw: data:image/raw-rgba;base64,)
//
// The reference compresses on the host with libjpeg (input JCS_EXT_RGBX, so alpha is
// dropped; jpeg_set_defaults, i.e. 2x2-subsampled chroma and the standard Huffman
// tables; quality 90 unless setJpegQuality changed it, clamped to 100).  Here the frame
// never leaves the GPU until it is text: one kernel drops alpha, nvJPEG encodes with the
// same subsampling, quality and table choice, the bitstream stays in device memory, a
// second kernel base64-encodes it, and one copy brings the text into pinned memory
// owned by the encoder.  Rows go out in frame order (row 0 = bottom first), as the
// reference hands its buffer to libjpeg.
//
// base64 follows boost's base64_from_binary<transform_width<const char*, 6, 8>>, which
// the reference uses: ceil(8n / 6) characters of the standard alphabet, the last one
// zero-filled in its low bits, and no '=' padding.
#include "../../include/isaac_b200.h"

#include <cuda_runtime.h>
#include <nvjpeg.h>

#include <cstring>
#include <string>

namespace isaacb
{
    void set_global_error(const std::string& msg);

    namespace
    {
        __constant__ char c_b64[64] = {'A', 'B', 'C', 'D', 'E', 'F', 'G', 'H', 'I', 'J', 'K', 'L', 'M', 'N', 'O', 'P',
                                       'Q', 'R', 'S', 'T', 'U', 'V', 'W', 'X', 'Y', 'Z', 'a', 'b', 'c', 'd', 'e', 'f',
                                       'g', 'h', 'i', 'j', 'k', 'l', 'm', 'n', 'o', 'p', 'q', 'r', 's', 't', 'u', 'v',
                                       'w', 'x', 'y', 'z', '0', '1', '2', '3', '4', '5', '6', '7', '8', '9', '+', '/'};

        // interleaved RGB from RGBA8 (alpha dropped, as JCS_EXT_RGBX reads the frame)
        __global__ void k_rgba_to_rgb(const uchar4* __restrict__ in, uint8_t* __restrict__ out, size_t n)
        {
            for(size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
            {
                const uchar4 p = __ldg(in + i);
                out[3 * i] = p.x;
                out[3 * i + 1] = p.y;
                out[3 * i + 2] = p.z;
            }
        }

        // one thread per 3-byte group: 4 characters, or 2 / 3 for a final group of 1 / 2 bytes
        __global__ void k_base64(const uint8_t* __restrict__ in, size_t n, char* __restrict__ out)
        {
            const size_t groups = (n + 2) / 3;
            for(size_t g = blockIdx.x * size_t(blockDim.x) + threadIdx.x; g < groups; g += size_t(gridDim.x) * blockDim.x)
            {
                const size_t i = 3 * g;
                const uint32_t b0 = __ldg(in + i);
                const uint32_t b1 = i + 1 < n ? __ldg(in + i + 1) : 0u;
                const uint32_t b2 = i + 2 < n ? __ldg(in + i + 2) : 0u;
                const uint32_t v = (b0 << 16) | (b1 << 8) | b2;
                const int chars = i + 2 < n ? 4 : (i + 1 < n ? 3 : 2);
                for(int k = 0; k < chars; ++k)
                    out[4 * g + k] = c_b64[(v >> (18 - 6 * k)) & 63u];
            }
        }

        size_t base64_chars(size_t n)
        {
            return (8 * n + 5) / 6;
        }

        unsigned grid_for(size_t n)
        {
            const size_t b = (n + 255) / 256;
            return unsigned(b < 4096 ? (b > 0 ? b : 1) : 4096);
        }

        const char* nvjpeg_name(nvjpegStatus_t s)
        {
            switch(s)
            {
            case NVJPEG_STATUS_SUCCESS: return "success";
            case NVJPEG_STATUS_NOT_INITIALIZED: return "not initialized";
            case NVJPEG_STATUS_INVALID_PARAMETER: return "invalid parameter";
            case NVJPEG_STATUS_BAD_JPEG: return "bad jpeg";
            case NVJPEG_STATUS_JPEG_NOT_SUPPORTED: return "jpeg not supported";
            case NVJPEG_STATUS_ALLOCATOR_FAILURE: return "allocator failure";
            case NVJPEG_STATUS_EXECUTION_FAILED: return "execution failed";
            case NVJPEG_STATUS_ARCH_MISMATCH: return "arch mismatch";
            case NVJPEG_STATUS_INTERNAL_ERROR: return "internal error";
            case NVJPEG_STATUS_IMPLEMENTATION_NOT_SUPPORTED: return "implementation not supported";
            default: return "unknown status";
            }
        }
    } // namespace
} // namespace isaacb

struct isaacb_encoder
{
    nvjpegHandle_t handle = nullptr;
    nvjpegEncoderState_t state = nullptr;
    nvjpegEncoderParams_t params = nullptr;
    uint32_t quality = 90; // IsaacCommunicator's jpeg_quality default
    uint8_t* rgb = nullptr; // device, interleaved RGB
    size_t rgbCap = 0;
    uint8_t* bits = nullptr; // device, JPEG bitstream
    size_t bitsCap = 0;
    char* text = nullptr; // device, base64 text
    size_t textCap = 0;
    char* host = nullptr; // pinned: the last message or JPEG
    size_t hostCap = 0;
};

namespace
{
    using isaacb::set_global_error;

    isaacb_status enc_fail(isaacb_status st, const std::string& m)
    {
        set_global_error(m);
        return st;
    }

    // device (or pinned host) buffer of at least `need` bytes, grown by doubling
    template<class T>
    bool grow(T*& p, size_t& cap, size_t need, bool pinned)
    {
        if(need <= cap && p)
            return true;
        size_t c = cap ? cap : 4096;
        while(c < need)
            c *= 2;
        void* q = nullptr;
        const cudaError_t e = pinned ? cudaHostAlloc(&q, c, cudaHostAllocDefault) : cudaMalloc(&q, c);
        if(e != cudaSuccess)
            return false;
        if(p)
            pinned ? cudaFreeHost(p) : cudaFree(p);
        p = static_cast<T*>(q);
        cap = c;
        return true;
    }

#define ISAACB_NVJPEG(call, what)                                                                                     \
    do                                                                                                                \
    {                                                                                                                 \
        const nvjpegStatus_t s_ = (call);                                                                             \
        if(s_ != NVJPEG_STATUS_SUCCESS)                                                                               \
            return enc_fail(ISAACB_CUDA_ERROR, std::string(what) + ": nvJPEG " + isaacb::nvjpeg_name(s_));            \
    } while(0)

    // JPEG of the frame into e->bits (device); the length in *len
    isaacb_status encode_jpeg_device(isaacb_encoder* e, const uint8_t* rgba, uint32_t w, uint32_t h, cudaStream_t s, size_t* len)
    {
        const size_t npix = size_t(w) * h;
        if(!grow(e->rgb, e->rgbCap, 3 * npix, false))
            return enc_fail(ISAACB_OOM, "isaacb_encode: RGB buffer");
        isaacb::k_rgba_to_rgb<<<isaacb::grid_for(npix), 256, 0, s>>>(reinterpret_cast<const uchar4*>(rgba), e->rgb, npix);
        cudaError_t ce = cudaGetLastError();
        if(ce != cudaSuccess)
            return enc_fail(ISAACB_CUDA_ERROR, std::string("isaacb_encode: ") + cudaGetErrorString(ce));
        nvjpegImage_t img{};
        img.channel[0] = e->rgb;
        img.pitch[0] = size_t(3) * w;
        ISAACB_NVJPEG(nvjpegEncoderParamsSetQuality(e->params, int(e->quality < 1 ? 1 : e->quality), s), "quality");
        ISAACB_NVJPEG(nvjpegEncodeImage(e->handle, e->state, e->params, &img, NVJPEG_INPUT_RGBI, int(w), int(h), s), "encode");
        size_t n = 0;
        ISAACB_NVJPEG(nvjpegEncodeRetrieveBitstreamDevice(e->handle, e->state, nullptr, &n, s), "bitstream length");
        if(!grow(e->bits, e->bitsCap, n, false))
            return enc_fail(ISAACB_OOM, "isaacb_encode: bitstream buffer");
        ISAACB_NVJPEG(nvjpegEncodeRetrieveBitstreamDevice(e->handle, e->state, e->bits, &n, s), "bitstream");
        *len = n;
        return ISAACB_OK;
    }
} // namespace

extern "C"
{
    isaacb_status isaacb_encoder_create(isaacb_encoder** out)
    {
        if(!out)
            return enc_fail(ISAACB_INVALID_ARG, "isaacb_encoder_create: null output");
        *out = nullptr;
        isaacb_encoder* e = new isaacb_encoder;
        nvjpegStatus_t s = nvjpegCreateSimple(&e->handle);
        if(s == NVJPEG_STATUS_SUCCESS)
            s = nvjpegEncoderStateCreate(e->handle, &e->state, nullptr);
        if(s == NVJPEG_STATUS_SUCCESS)
            s = nvjpegEncoderParamsCreate(e->handle, &e->params, nullptr);
        // jpeg_set_defaults: 2x2 chroma subsampling, baseline, standard Huffman tables
        if(s == NVJPEG_STATUS_SUCCESS)
            s = nvjpegEncoderParamsSetSamplingFactors(e->params, NVJPEG_CSS_420, nullptr);
        if(s == NVJPEG_STATUS_SUCCESS)
            s = nvjpegEncoderParamsSetOptimizedHuffman(e->params, 0, nullptr);
        if(s != NVJPEG_STATUS_SUCCESS)
        {
            isaacb_encoder_destroy(e);
            return enc_fail(ISAACB_CUDA_ERROR, std::string("isaacb_encoder_create: nvJPEG ") + isaacb::nvjpeg_name(s));
        }
        *out = e;
        return ISAACB_OK;
    }

    isaacb_status isaacb_encoder_destroy(isaacb_encoder* e)
    {
        if(!e)
            return ISAACB_OK;
        if(e->params)
            nvjpegEncoderParamsDestroy(e->params);
        if(e->state)
            nvjpegEncoderStateDestroy(e->state);
        if(e->handle)
            nvjpegDestroy(e->handle);
        cudaFree(e->rgb);
        cudaFree(e->bits);
        cudaFree(e->text);
        if(e->host)
            cudaFreeHost(e->host);
        delete e;
        return ISAACB_OK;
    }

    isaacb_status isaacb_encoder_set_quality(isaacb_encoder* e, uint32_t quality)
    {
        if(!e)
            return enc_fail(ISAACB_INVALID_ARG, "isaacb_encoder_set_quality: null encoder");
        e->quality = quality > 100 ? 100 : quality;
        return ISAACB_OK;
    }

    isaacb_status isaacb_encoder_get_quality(const isaacb_encoder* e, uint32_t* quality)
    {
        if(!e || !quality)
            return enc_fail(ISAACB_INVALID_ARG, "isaacb_encoder_get_quality: null argument");
        *quality = e->quality;
        return ISAACB_OK;
    }

    isaacb_status isaacb_encode_jpeg(
        isaacb_encoder* e,
        const uint8_t* rgba,
        uint32_t width,
        uint32_t height,
        void* stream,
        const uint8_t** jpeg,
        size_t* length)
    {
        if(!e || !rgba || !jpeg || !length || width == 0 || height == 0 || width > 16384 || height > 16384)
            return enc_fail(ISAACB_INVALID_ARG, "isaacb_encode_jpeg: bad arguments");
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        size_t n = 0;
        const isaacb_status st = encode_jpeg_device(e, rgba, width, height, s, &n);
        if(st != ISAACB_OK)
            return st;
        if(!grow(e->host, e->hostCap, n + 1, true))
            return enc_fail(ISAACB_OOM, "isaacb_encode_jpeg: pinned buffer");
        cudaError_t ce = cudaMemcpyAsync(e->host, e->bits, n, cudaMemcpyDeviceToHost, s);
        if(ce == cudaSuccess)
            ce = cudaStreamSynchronize(s);
        if(ce != cudaSuccess)
            return enc_fail(ISAACB_CUDA_ERROR, std::string("isaacb_encode_jpeg: ") + cudaGetErrorString(ce));
        *jpeg = reinterpret_cast<const uint8_t*>(e->host);
        *length = n;
        return ISAACB_OK;
    }

    isaacb_status isaacb_encode_frame(
        isaacb_encoder* e,
        const uint8_t* rgba,
        uint32_t width,
        uint32_t height,
        int32_t jpeg,
        void* stream,
        const char** message,
        size_t* length)
    {
        if(!e || !rgba || !message || !length || width == 0 || height == 0 || width > 16384 || height > 16384)
            return enc_fail(ISAACB_INVALID_ARG, "isaacb_encode_frame: bad arguments");
        const cudaStream_t s = static_cast<cudaStream_t>(stream);
        const uint8_t* bytes = rgba;
        size_t n = size_t(width) * height * 4;
        if(jpeg)
        {
            const isaacb_status st = encode_jpeg_device(e, rgba, width, height, s, &n);
            if(st != ISAACB_OK)
                return st;
            bytes = e->bits;
        }
        static const char kHeadJpeg[] = "{\"payload\": \"data:image/jpeg;base64,";
        static const char kHeadRaw[] = "{\"payload\": \"data:image/raw-rgba;base64,";
        static const char kFoot[] = "\"}";
        const char* head = jpeg ? kHeadJpeg : kHeadRaw;
        const size_t hl = std::strlen(head), fl = std::strlen(kFoot);
        const size_t chars = isaacb::base64_chars(n);
        if(!grow(e->text, e->textCap, chars, false) || !grow(e->host, e->hostCap, hl + chars + fl + 1, true))
            return enc_fail(ISAACB_OOM, "isaacb_encode_frame: text buffers");
        isaacb::k_base64<<<isaacb::grid_for((n + 2) / 3), 256, 0, s>>>(bytes, n, e->text);
        cudaError_t ce = cudaGetLastError();
        if(ce == cudaSuccess)
            ce = cudaMemcpyAsync(e->host + hl, e->text, chars, cudaMemcpyDeviceToHost, s);
        if(ce == cudaSuccess)
            ce = cudaStreamSynchronize(s);
        if(ce != cudaSuccess)
            return enc_fail(ISAACB_CUDA_ERROR, std::string("isaacb_encode_frame: ") + cudaGetErrorString(ce));
        std::memcpy(e->host, head, hl);
        std::memcpy(e->host + hl + chars, kFoot, fl + 1);
        *message = e->host;
        *length = hl + chars + fl;
        return ISAACB_OK;
    }

    isaacb_status isaacb_base64(const uint8_t* in, size_t n, char* out, void* stream)
    {
        if((!in || !out) && n > 0)
            return enc_fail(ISAACB_INVALID_ARG, "isaacb_base64: null buffer");
        if(n == 0)
            return ISAACB_OK;
        isaacb::k_base64<<<isaacb::grid_for((n + 2) / 3), 256, 0, static_cast<cudaStream_t>(stream)>>>(in, n, out);
        const cudaError_t ce = cudaGetLastError();
        if(ce != cudaSuccess)
            return enc_fail(ISAACB_CUDA_ERROR, std::string("isaacb_base64: ") + cudaGetErrorString(ce));
        return ISAACB_OK;
    }
}
