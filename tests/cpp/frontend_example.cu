// Simulation-side use of the C++ front end (include/isaac_b200.hpp), in the shape
// of the reference's example (example/example.cpp:36-228): a scalar source read in
// place (linearData), a vector source read only through its device operator[], and
// a particle source behind getIterator(cell).  Reads a scene file, renders one
// frame, writes the frame and the per-source min/max.  With --field the vector source
// is a field source (the reference's FieldSourceList) with advection, and the frame
// written is the third of three.
//
// usage: frontend_example <scene.bin> <out.bin> [--field]
#include "isaac_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

using isaacb::float_dim;
using isaacb::int3v;
using isaacb::uint3v;

struct ScalarSource
{
    static const int featureDim = 1;
    static const int guardSize = 0;
    static const bool persistent = true;
    const float* ptr;
    int X, Y;
    static const char* getName() { return "scalar"; }
    void update(bool, void*) {}
    const float* linearData() const { return ptr; }
    __host__ __device__ float_dim<1> operator[](const int3v& c) const { return {ptr[c.x + c.y * X + c.z * X * Y]}; }
};

struct VectorSource
{
    static const int featureDim = 3;
    static const int guardSize = 0;
    static const bool persistent = true;
    const float* ptr;
    int X, Y;
    static const char* getName() { return "vector"; }
    void update(bool, void*) {}
    __host__ __device__ float_dim<3> operator[](const int3v& c) const
    {
        const float* p = ptr + 3 * (size_t(c.x) + size_t(c.y) * X + size_t(c.z) * X * Y);
        return {p[0], p[1], p[2]};
    }
};

struct CellIterator
{
    size_t size;
    const float* pos;
    const float* attr;
    __host__ __device__ void next()
    {
        pos += 3;
        attr += 3;
    }
    __host__ __device__ float_dim<3> getPosition() const { return {pos[0], pos[1], pos[2]}; }
    __host__ __device__ float_dim<3> getAttribute() const { return {attr[0], attr[1], attr[2]}; }
    __host__ __device__ float getRadius() const { return 0.45f; }
};

struct ParticleSourceCells
{
    static const int featureDim = 3;
    const unsigned* offsets;
    const float* pos;
    const float* attr;
    int PX, PY;
    static const char* getName() { return "particles"; }
    void update(bool, void*) {}
    __host__ __device__ CellIterator getIterator(const uint3v& c) const
    {
        const size_t i = size_t(c.x) + size_t(c.y) * PX + size_t(c.z) * PX * PY;
        const unsigned b = offsets[i], e = offsets[i + 1];
        return CellIterator{size_t(e - b), pos + 3 * size_t(b), attr + 3 * size_t(b)};
    }
};

template<class T>
static T* upload(const std::vector<T>& h)
{
    T* d = nullptr;
    cudaMalloc(&d, h.size() * sizeof(T));
    cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    return d;
}

template<bool Field>
int run(ScalarSource& sc, VectorSource& ve, ParticleSourceCells& ps, int n, int W, int H, int PX, int PY, int PZ,
        const std::array<double, 16>& P, const std::array<double, 16>& MV, const char* outPath);

int main(int argc, char** argv)
{
    if(argc < 3)
        return 2;
    FILE* f = fopen(argv[1], "rb");
    if(!f)
        return 3;
    int hdr[6]; // n, W, H, PX, PY, PZ
    if(fread(hdr, sizeof(int), 6, f) != 6)
        return 4;
    const int n = hdr[0], W = hdr[1], H = hdr[2], PX = hdr[3], PY = hdr[4], PZ = hdr[5];
    std::array<double, 16> P, MV;
    fread(P.data(), sizeof(double), 16, f);
    fread(MV.data(), sizeof(double), 16, f);
    const size_t nv = size_t(n) * n * n, ncell = size_t(PX) * PY * PZ;
    std::vector<float> scalar(nv), vec(3 * nv);
    fread(scalar.data(), sizeof(float), nv, f);
    fread(vec.data(), sizeof(float), 3 * nv, f);
    std::vector<unsigned> off(ncell + 1);
    fread(off.data(), sizeof(unsigned), ncell + 1, f);
    const size_t np = off[ncell];
    std::vector<float> pos(3 * np), attr(3 * np);
    fread(pos.data(), sizeof(float), 3 * np, f);
    fread(attr.data(), sizeof(float), 3 * np, f);
    fclose(f);

    ScalarSource sc{upload(scalar), n, n};
    VectorSource ve{upload(vec), n, n};
    ParticleSourceCells ps{upload(off), upload(pos), upload(attr), PX, PY};
    const bool field = argc > 3 && std::string(argv[3]) == "--field";
    return field ? run<true>(sc, ve, ps, n, W, H, PX, PY, PZ, P, MV, argv[2])
                 : run<false>(sc, ve, ps, n, W, H, PX, PY, PZ, P, MV, argv[2]);
}

template<bool Field, class Volumes, class Fields, class Particles>
static int render(Volumes& volumes, Fields& fields, Particles& particles, int n, int W, int H, int PX, int PY, int PZ,
                  const std::array<double, 16>& P, const std::array<double, 16>& MV, const char* outPath)
{
    using Viz = isaacb::IsaacVisualization<Volumes, Fields, Particles>;
    Viz viz(
        "frontend",
        {uint32_t(W), uint32_t(H)},
        {uint32_t(n), uint32_t(n), uint32_t(n)},
        {uint32_t(n), uint32_t(n), uint32_t(n)},
        {uint32_t(PX), uint32_t(PY), uint32_t(PZ)},
        {0, 0, 0},
        volumes,
        fields,
        particles);
    viz.functions[1].source = "length";
    viz.functions[2].source = "length";
    viz.updateFunctions();
    viz.transferPoints[0] = {{0, {0, 0, 0, 0}}, {300, {0.8f, 0.3f, 0.2f, 0.1f}}, {700, {0.2f, 0.7f, 0.9f, 0.4f}}, {1024, {1, 1, 0.5f, 0.9f}}};
    viz.transferPoints[1] = {{0, {0, 0, 0, 0}}, {1024, {0.3f, 0.9f, 0.4f, 0.6f}}};
    viz.transferPoints[2] = {{0, {0.1f, 0.9f, 0.1f, 1}}, {1024, {0.9f, 0.1f, 0.1f, 1}}};
    viz.updateTransfer();
    viz.setInterpolation(true);
    viz.setIsoThreshold(0, 0.45f);
    viz.setCamera(P, MV);
    const uint8_t* frame = nullptr;
    if(Field)
    {
        viz.setAdvection(1.0f, 0.95f, 1, 1, 40);
        for(int k = 0; k < 3; ++k)
            frame = viz.doVisualization();
    }
    else
        frame = viz.doVisualization();
    auto mm = viz.minMax();
    FILE* o = fopen(outPath, "wb");
    fwrite(frame, 1, size_t(W) * H * 4, o);
    fwrite(mm.first.data(), sizeof(float), 3, o);
    fwrite(mm.second.data(), sizeof(float), 3, o);
    fclose(o);
    printf("frontend ok\n");
    return 0;
}

template<bool Field>
int run(ScalarSource& sc, VectorSource& ve, ParticleSourceCells& ps, int n, int W, int H, int PX, int PY, int PZ,
        const std::array<double, 16>& P, const std::array<double, 16>& MV, const char* outPath)
{
    std::tuple<ParticleSourceCells> particles{ps};
    if constexpr(Field)
    {
        std::tuple<ScalarSource> volumes{sc};
        std::tuple<VectorSource> fields{ve};
        return render<true>(volumes, fields, particles, n, W, H, PX, PY, PZ, P, MV, outPath);
    }
    else
    {
        std::tuple<ScalarSource, VectorSource> volumes{sc, ve};
        std::tuple<> fields;
        return render<false>(volumes, fields, particles, n, W, H, PX, PY, PZ, P, MV, outPath);
    }
}
