// Output side of a render: the float RGBA frame turned into files.
//
//   * 8-bit RGBA on the device with the arithmetic of XTracer's PNG writer
//     (lib/nimg/img.cc:150-172): each channel times 255, clamped at 255,
//     truncated (a NaN channel gives 0, as the reference's float to unsigned
//     char conversion does on x86-64);
//   * PNG: 8-bit RGBA, one zlib stream, filter type 0 on every row (the pixels
//     equal those of stbi_write_png on the same frame; the compressed bytes may
//     differ);
//   * OpenEXR: uncompressed scanlines, float channels B, G, R, as XTracer's EXR
//     writer asks tinyexr for (img.cc:72-141).
#include <zlib.h>

#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "xtgpu_internal.cuh"

namespace xtg {
namespace {

__device__ __forceinline__ unsigned char channel8(float v)
{
    const float s = v * 255.f;
    if (!(s == s) || s <= 0.f) return 0;   // NaN; colours are clamped at 0 before
    return (unsigned char)(s > 255.f ? 255.f : s);
}

__global__ void k_rgba8(const float4 *__restrict__ f, int64_t n, uchar4 *__restrict__ o)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 c = f[i];
        o[i] = make_uchar4(channel8(c.x), channel8(c.y), channel8(c.z), channel8(c.w));
    }
}

void put_be32(std::vector<unsigned char> &v, uint32_t x)
{
    v.push_back((unsigned char)(x >> 24));
    v.push_back((unsigned char)(x >> 16));
    v.push_back((unsigned char)(x >> 8));
    v.push_back((unsigned char)x);
}

void png_chunk(std::vector<unsigned char> &out, const char type[4], const unsigned char *data, size_t n)
{
    put_be32(out, (uint32_t)n);
    const size_t at = out.size();
    out.insert(out.end(), type, type + 4);
    if (n) out.insert(out.end(), data, data + n);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, out.data() + at, (uInt)(4 + n));
    put_be32(out, (uint32_t)crc);
}

template <typename T>
void put_le(std::vector<unsigned char> &v, T x)
{
    unsigned char b[sizeof(T)];
    memcpy(b, &x, sizeof(T));
    v.insert(v.end(), b, b + sizeof(T));
}

void put_str(std::vector<unsigned char> &v, const char *s) { v.insert(v.end(), s, s + strlen(s) + 1); }

void exr_attr(std::vector<unsigned char> &v, const char *name, const char *type, const std::vector<unsigned char> &val)
{
    put_str(v, name);
    put_str(v, type);
    put_le<int32_t>(v, (int32_t)val.size());
    v.insert(v.end(), val.begin(), val.end());
}

xtgpu_status write_file(const char *path, const std::vector<unsigned char> &bytes, const char *what)
{
    FILE *f = fopen(path, "wb");
    if (!f) {
        set_error(std::string(what) + ": cannot open " + path);
        return XTGPU_ERR_INVALID;
    }
    const size_t n = fwrite(bytes.data(), 1, bytes.size(), f);
    const int closed = fclose(f);
    if (n != bytes.size() || closed != 0) {
        set_error(std::string(what) + ": write failed for " + path);
        return XTGPU_ERR_INVALID;
    }
    return XTGPU_OK;
}

}  // namespace
}  // namespace xtg

using namespace xtg;

extern "C" {

xtgpu_status xtgpu_frame_rgba8(const float *rgba_dev, int64_t n_pixels, uint8_t *rgba8_dev, void *stream)
{
    if (n_pixels < 0 || (n_pixels && (!rgba_dev || !rgba8_dev))) {
        set_error("xtgpu_frame_rgba8: bad argument");
        return XTGPU_ERR_INVALID;
    }
    if (n_pixels == 0) return XTGPU_OK;
    const int blocks = (int)std::min<int64_t>((n_pixels + 255) / 256, 148 * 16);
    k_rgba8<<<blocks, 256, 0, (cudaStream_t)stream>>>((const float4 *)rgba_dev, n_pixels, (uchar4 *)rgba8_dev);
    XTG_CUDA(cudaGetLastError());
    return XTGPU_OK;
}

xtgpu_status xtgpu_write_png(const char *path, int32_t width, int32_t height, const uint8_t *rgba8_host)
{
    if (!path || !rgba8_host || width <= 0 || height <= 0 || (int64_t)width * height > (1ll << 31)) {
        set_error("xtgpu_write_png: bad argument");
        return XTGPU_ERR_INVALID;
    }
    const size_t row = 1 + 4 * (size_t)width;
    std::vector<unsigned char> raw(row * (size_t)height);
    for (int32_t y = 0; y < height; ++y) {
        raw[row * y] = 0;   // filter type 0 (none)
        memcpy(&raw[row * y + 1], rgba8_host + 4 * (size_t)width * y, 4 * (size_t)width);
    }
    uLongf zn = compressBound((uLong)raw.size());
    std::vector<unsigned char> z(zn);
    if (compress2(z.data(), &zn, raw.data(), (uLong)raw.size(), 6) != Z_OK) {
        set_error("xtgpu_write_png: zlib compression failed");
        return XTGPU_ERR_INVALID;
    }
    std::vector<unsigned char> out = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    std::vector<unsigned char> ihdr;
    put_be32(ihdr, (uint32_t)width);
    put_be32(ihdr, (uint32_t)height);
    const unsigned char tail[5] = {8, 6, 0, 0, 0};   // 8 bits, RGBA, deflate, filter 0, no interlace
    ihdr.insert(ihdr.end(), tail, tail + 5);
    png_chunk(out, "IHDR", ihdr.data(), ihdr.size());
    png_chunk(out, "IDAT", z.data(), zn);
    png_chunk(out, "IEND", nullptr, 0);
    return write_file(path, out, "xtgpu_write_png");
}

xtgpu_status xtgpu_write_exr(const char *path, int32_t width, int32_t height, const float *rgba_host)
{
    if (!path || !rgba_host || width <= 0 || height <= 0 || (int64_t)width * height > (1ll << 31)) {
        set_error("xtgpu_write_exr: bad argument");
        return XTGPU_ERR_INVALID;
    }
    std::vector<unsigned char> v = {0x76, 0x2f, 0x31, 0x01};   // magic
    put_le<int32_t>(v, 2);                                     // version 2, single-part scanline
    std::vector<unsigned char> ch;
    for (const char *name : {"B", "G", "R"}) {                 // channels in alphabetical order
        put_str(ch, name);
        put_le<int32_t>(ch, 2);                                // FLOAT
        put_le<int32_t>(ch, 0);                                // pLinear + reserved
        put_le<int32_t>(ch, 1);                                // x sampling
        put_le<int32_t>(ch, 1);                                // y sampling
    }
    ch.push_back(0);
    exr_attr(v, "channels", "chlist", ch);
    exr_attr(v, "compression", "compression", {0});           // NO_COMPRESSION
    std::vector<unsigned char> box;
    for (int32_t x : {0, 0, width - 1, height - 1}) put_le<int32_t>(box, x);
    exr_attr(v, "dataWindow", "box2i", box);
    exr_attr(v, "displayWindow", "box2i", box);
    exr_attr(v, "lineOrder", "lineOrder", {0});               // INCREASING_Y
    std::vector<unsigned char> one;
    put_le<float>(one, 1.f);
    exr_attr(v, "pixelAspectRatio", "float", one);
    std::vector<unsigned char> center;
    put_le<float>(center, 0.f);
    put_le<float>(center, 0.f);
    exr_attr(v, "screenWindowCenter", "v2f", center);
    exr_attr(v, "screenWindowWidth", "float", one);
    v.push_back(0);                                            // end of header
    // offset table, then one scanline per block: y, size, B row, G row, R row
    const size_t block = 8 + 3 * 4 * (size_t)width;
    const size_t table = v.size();
    for (int32_t y = 0; y < height; ++y) put_le<uint64_t>(v, (uint64_t)(table + 8 * (size_t)height + block * y));
    std::vector<float> rowf((size_t)width);
    for (int32_t y = 0; y < height; ++y) {
        put_le<int32_t>(v, y);
        put_le<int32_t>(v, (int32_t)(3 * 4 * (size_t)width));
        for (int c : {2, 1, 0}) {
            for (int32_t x = 0; x < width; ++x) rowf[x] = rgba_host[4 * ((size_t)width * y + x) + c];
            const unsigned char *b = (const unsigned char *)rowf.data();
            v.insert(v.end(), b, b + 4 * (size_t)width);
        }
    }
    return write_file(path, v, "xtgpu_write_exr");
}

xtgpu_status xtgpu_save_png_host(const char *path, int32_t width, int32_t height, const float *rgba_host,
                                 void *stream)
{
    if (!path || !rgba_host || width <= 0 || height <= 0) {
        set_error("xtgpu_save_png_host: bad argument");
        return XTGPU_ERR_INVALID;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = (int64_t)width * height;
    float *f = nullptr;
    uint8_t *q = nullptr;
    XTG_CUDA(cudaMallocAsync((void **)&f, sizeof(float) * 4 * n, s));
    cudaError_t e = cudaMallocAsync((void **)&q, 4 * (size_t)n, s);
    std::vector<uint8_t> host(4 * (size_t)n);
    xtgpu_status st = XTGPU_OK;
    if (e == cudaSuccess) e = cudaMemcpyAsync(f, rgba_host, sizeof(float) * 4 * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) st = xtgpu_frame_rgba8(f, n, q, stream);
    if (e == cudaSuccess && st == XTGPU_OK) e = cudaMemcpyAsync(host.data(), q, 4 * (size_t)n, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess && st == XTGPU_OK) e = cudaStreamSynchronize(s);
    if (f) cudaFreeAsync(f, s);
    if (q) cudaFreeAsync(q, s);
    if (e != cudaSuccess) return cuda_fail(e, "xtgpu_save_png_host", __FILE__, __LINE__);
    if (st != XTGPU_OK) return st;
    return xtgpu_write_png(path, width, height, host.data());
}

// raygraph::write (util/raygraph.cc:8-75) of two-sample paths: the ply header,
// per path the origin with the default ColorRGBAf (0, 0, 0) and the hit point
// with its colour, then one edge per path.  Positions print as the doubles the
// reference holds (Vector3f), colours as floats, through an ostream with its
// default format, as the reference writes them.
xtgpu_status xtgpu_write_raygraph_ply(const char *path, int64_t n_paths, const float *records)
{
    if (!path || n_paths < 0 || (n_paths && !records)) {
        set_error("xtgpu_write_raygraph_ply: bad argument");
        return XTGPU_ERR_INVALID;
    }
    std::ofstream file(path);
    if (!file) {
        set_error(std::string("xtgpu_write_raygraph_ply: cannot open ") + path);
        return XTGPU_ERR_INVALID;
    }
    file << "ply" << std::endl;
    file << "format ascii 1.0" << std::endl;
    file << "comment object: A single line" << std::endl;
    file << "element vertex " << (size_t)(2 * n_paths) << std::endl;
    file << "property float x" << std::endl;
    file << "property float y" << std::endl;
    file << "property float z" << std::endl;
    file << "property float red" << std::endl;
    file << "property float green" << std::endl;
    file << "property float blue" << std::endl;
    file << "element edge " << (size_t)n_paths << std::endl;
    file << "property int vertex1" << std::endl;
    file << "property int vertex2" << std::endl;
    file << "end_header" << std::endl;
    const float zero = 0.f;
    for (int64_t i = 0; i < n_paths; ++i) {
        const float *r = records + 10 * i;
        file << (double)r[0] << " " << (double)r[1] << " " << (double)r[2] << " " << zero << " " << zero << " "
             << zero << std::endl;
        file << (double)r[3] << " " << (double)r[4] << " " << (double)r[5] << " " << r[6] << " " << r[7] << " "
             << r[8] << std::endl;
    }
    for (int64_t i = 0; i < n_paths; ++i) file << (size_t)(2 * i) << " " << (size_t)(2 * i + 1) << std::endl;
    file.close();
    if (!file) {
        set_error(std::string("xtgpu_write_raygraph_ply: write failed: ") + path);
        return XTGPU_ERR_CUDA;
    }
    return XTGPU_OK;
}

}  // extern "C"
