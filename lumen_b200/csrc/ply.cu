/*
 * ply.cu - Gaussian PLY scenes into the SoA layout (include/lumen_ply.h).
 *
 * The header is parsed on the host; columns are found by property name.
 * Binary little-endian vertex data whose mapped properties are 4-byte
 * aligned goes to the device raw, in chunks through two page-locked buffers
 * (the next chunk is read from the file while the previous one is copied and
 * de-interleaved), and ply_deinterleave_kernel scatters each vertex into the
 * SoA arrays, transposing the channel-major f_rest block into
 * sh[k * 3 + ch]. ASCII files (and unaligned binary ones) are parsed on the
 * host and uploaded.
 */
#include <algorithm>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "splat_common.cuh"
#include "../../include/lumen_ply.h"

namespace lumen {
LumenStatus map_cuda(cudaError_t e);

namespace {

constexpr int kMaxRestPerChannel = 15;

struct Prop {
    std::string name;
    int size = 0;          /* bytes in a binary file */
    bool is_f32 = false;
    int offset = 0;        /* byte offset in a binary vertex */
};

struct Layout {
    int64_t count = 0;
    bool binary = false;
    int stride = 0;
    int64_t data_offset = 0;
    std::vector<Prop> props;
    /* property indices; -1 when absent */
    int pos[3] = {-1, -1, -1}, scl[3] = {-1, -1, -1}, rot[4] = {-1, -1, -1, -1}, op = -1, dc[3] = {-1, -1, -1};
    int rest_per_ch = 0;   /* f_rest count / 3, at most 15 */
    std::vector<int> rest; /* f_rest_j -> property index */
    bool log_values = false;
};

int type_size(const std::string& t, bool* is_f32) {
    *is_f32 = false;
    if (t == "char" || t == "int8" || t == "uchar" || t == "uint8") return 1;
    if (t == "short" || t == "int16" || t == "ushort" || t == "uint16") return 2;
    if (t == "int" || t == "int32" || t == "uint" || t == "uint32") return 4;
    if (t == "float" || t == "float32") { *is_f32 = true; return 4; }
    if (t == "double" || t == "float64") return 8;
    return -1;
}

LumenStatus parse_header(FILE* fp, int values, Layout* L) {
    char line[1024];
    if (!fgets(line, sizeof line, fp)) return LUMEN_ERROR_IO_FAILURE;
    if (strncmp(line, "ply", 3) != 0) return LUMEN_ERROR_INVALID_ARGUMENT;
    bool in_vertex = false, seen_vertex = false, have_format = false;
    int lines = 0;
    for (;;) {
        if (!fgets(line, sizeof line, fp)) return LUMEN_ERROR_INVALID_ARGUMENT;   /* no end_header */
        if (++lines > 100000) return LUMEN_ERROR_INVALID_ARGUMENT;
        char a[256] = {0}, b[256] = {0}, c[256] = {0}, d[256] = {0};
        const int n = sscanf(line, "%255s %255s %255s %255s", a, b, c, d);
        if (n <= 0) continue;
        const std::string w = a;
        if (w == "end_header") break;
        if (w == "comment" || w == "obj_info") continue;
        if (w == "format") {
            if (n < 2) return LUMEN_ERROR_INVALID_ARGUMENT;
            if (!strcmp(b, "ascii")) L->binary = false;
            else if (!strcmp(b, "binary_little_endian")) L->binary = true;
            else return LUMEN_ERROR_INVALID_ARGUMENT;   /* big-endian */
            have_format = true;
        } else if (w == "element") {
            if (n < 3) return LUMEN_ERROR_INVALID_ARGUMENT;
            if (!strcmp(b, "vertex")) {
                if (seen_vertex) return LUMEN_ERROR_INVALID_ARGUMENT;
                char* end = nullptr;
                errno = 0;
                const long long cnt = strtoll(c, &end, 10);
                if (errno || cnt < 0 || cnt >= (1ll << 31)) return LUMEN_ERROR_INVALID_ARGUMENT;
                L->count = cnt;
                in_vertex = seen_vertex = true;
            } else {
                /* an element before the vertices would shift their data */
                if (!seen_vertex) return LUMEN_ERROR_INVALID_ARGUMENT;
                in_vertex = false;
            }
        } else if (w == "property") {
            if (!in_vertex) continue;
            if (n < 3 || !strcmp(b, "list")) return LUMEN_ERROR_INVALID_ARGUMENT;
            Prop p;
            p.name = c;
            p.size = type_size(b, &p.is_f32);
            if (p.size < 0) return LUMEN_ERROR_INVALID_ARGUMENT;
            p.offset = L->stride;
            L->stride += p.size;
            L->props.push_back(p);
        }
    }
    if (!have_format || !seen_vertex) return LUMEN_ERROR_INVALID_ARGUMENT;
    L->data_offset = (int64_t)ftell(fp);
    /* columns by name */
    std::vector<int> rest_idx;
    for (int i = 0; i < (int)L->props.size(); ++i) {
        const std::string& nm = L->props[(size_t)i].name;
        static const char* pos_names[3] = {"x", "y", "z"};
        for (int k = 0; k < 3; ++k) {
            if (nm == pos_names[k]) L->pos[k] = i;
            if (nm == "scale_" + std::to_string(k)) L->scl[k] = i;
            if (nm == "f_dc_" + std::to_string(k)) L->dc[k] = i;
        }
        for (int k = 0; k < 4; ++k)
            if (nm == "rot_" + std::to_string(k)) L->rot[k] = i;
        if (nm == "opacity") L->op = i;
        if (nm.compare(0, 7, "f_rest_") == 0) {
            char* end = nullptr;
            const long j = strtol(nm.c_str() + 7, &end, 10);
            if (end && *end == 0 && j >= 0 && j < 3 * kMaxRestPerChannel) {
                if ((int)rest_idx.size() <= j) rest_idx.resize((size_t)j + 1, -1);
                rest_idx[(size_t)j] = i;
            }
        }
    }
    int mapped[14] = {L->pos[0], L->pos[1], L->pos[2], L->scl[0], L->scl[1], L->scl[2], L->rot[0],
                      L->rot[1], L->rot[2], L->rot[3], L->op, L->dc[0], L->dc[1], L->dc[2]};
    for (int k = 0; k < 14; ++k) {
        if (mapped[k] < 0) return LUMEN_ERROR_INVALID_ARGUMENT;
        if (L->binary && !L->props[(size_t)mapped[k]].is_f32) return LUMEN_ERROR_INVALID_ARGUMENT;
    }
    /* the leading run f_rest_0 .. f_rest_{3m-1}, all present */
    int run = 0;
    while (run < (int)rest_idx.size() && rest_idx[(size_t)run] >= 0 &&
           (!L->binary || L->props[(size_t)rest_idx[(size_t)run]].is_f32))
        ++run;
    L->rest_per_ch = run / 3;
    L->rest.assign(rest_idx.begin(), rest_idx.begin() + 3 * L->rest_per_ch);
    L->log_values = values == LUMEN_PLY_VALUES_LOG || (values == LUMEN_PLY_VALUES_AUTO && L->rest_per_ch > 0);
    return LUMEN_SUCCESS;
}

int sh_degree_of(int rest_per_ch) {
    if (rest_per_ch >= 15) return 3;
    if (rest_per_ch >= 8) return 2;
    if (rest_per_ch >= 3) return 1;
    return 0;
}

void fill_info(const Layout& L, LumenPlyInfo* info) {
    if (!info) return;
    info->count = L.count;
    info->binary = L.binary ? 1 : 0;
    info->sh_degree = sh_degree_of(L.rest_per_ch);
    info->log_values = L.log_values ? 1 : 0;
    info->vertex_stride = L.stride;
    info->data_offset = L.data_offset;
}

/* One vertex's values (by property index) into the SoA arrays at slot i. */
void store_vertex(const Layout& L, const float* v, int64_t i, float* means, float* scales, float* quats,
                  float* opacities, float* sh) {
    for (int k = 0; k < 3; ++k) {
        means[i * 3 + k] = v[L.pos[k]];
        scales[i * 3 + k] = v[L.scl[k]];
    }
    for (int k = 0; k < 4; ++k) quats[i * 4 + k] = v[L.rot[k]];
    opacities[i] = v[L.op];
    float* s = sh + i * 48;
    for (int ch = 0; ch < 3; ++ch) s[ch] = v[L.dc[ch]];
    for (int k = 1; k < 16; ++k)
        for (int ch = 0; ch < 3; ++ch)
            s[k * 3 + ch] = k - 1 < L.rest_per_ch ? v[L.rest[(size_t)(ch * L.rest_per_ch + k - 1)]] : 0.0f;
}

float read_prop(const unsigned char* row, const Prop& p) {
    /* little-endian host; every type read as its value converted to float */
    float f = 0.0f;
    if (p.is_f32) { memcpy(&f, row + p.offset, 4); return f; }
    return 0.0f;   /* unmapped properties of other types are never read */
}

/* Host path for both formats: vertices in order into SoA. */
LumenStatus load_host(FILE* fp, const Layout& L, float* means, float* scales, float* quats, float* opacities,
                      float* sh) {
    std::vector<float> v(L.props.size());
    if (L.binary) {
        const int64_t rows = 4096;
        std::vector<unsigned char> buf((size_t)(rows * L.stride));
        for (int64_t i0 = 0; i0 < L.count; i0 += rows) {
            const int64_t nr = L.count - i0 < rows ? L.count - i0 : rows;
            if (fread(buf.data(), (size_t)L.stride, (size_t)nr, fp) != (size_t)nr) return LUMEN_ERROR_IO_FAILURE;
            for (int64_t r = 0; r < nr; ++r) {
                const unsigned char* row = buf.data() + r * L.stride;
                for (size_t k = 0; k < L.props.size(); ++k) v[k] = read_prop(row, L.props[k]);
                store_vertex(L, v.data(), i0 + r, means, scales, quats, opacities, sh);
            }
        }
        return LUMEN_SUCCESS;
    }
    std::string line;
    line.reserve(4096);
    for (int64_t i = 0; i < L.count; ++i) {
        line.clear();
        int ch;
        while ((ch = fgetc(fp)) != EOF && ch != '\n') line.push_back((char)ch);
        if (line.empty() && ch == EOF) return LUMEN_ERROR_IO_FAILURE;
        const char* p = line.c_str();
        for (size_t k = 0; k < L.props.size(); ++k) {
            char* end = nullptr;
            v[k] = strtof(p, &end);
            if (end == p) return LUMEN_ERROR_INVALID_ARGUMENT;   /* fewer values than properties */
            p = end;
        }
        store_vertex(L, v.data(), i, means, scales, quats, opacities, sh);
    }
    return LUMEN_SUCCESS;
}

/* Byte offsets of the mapped float32 columns of a binary vertex. */
struct PlyColumns {
    int stride;
    int pos[3], scl[3], rot[4], op, dc[3];
    int rest_per_ch;
    int rest[3 * kMaxRestPerChannel];
};

__global__ void ply_deinterleave_kernel(const unsigned char* __restrict__ rows, long long n, long long first,
                                        PlyColumns c, float* means, float* scales, float* quats, float* opacities,
                                        float* sh) {
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += nthreads) {
        const unsigned char* row = rows + r * c.stride;
        auto f = [&](int off) { return *reinterpret_cast<const float*>(row + off); };
        const long long i = first + r;
        for (int k = 0; k < 3; ++k) {
            means[i * 3 + k] = f(c.pos[k]);
            scales[i * 3 + k] = f(c.scl[k]);
        }
        reinterpret_cast<float4*>(quats)[i] = make_float4(f(c.rot[0]), f(c.rot[1]), f(c.rot[2]), f(c.rot[3]));
        opacities[i] = f(c.op);
        float v[48];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) v[ch] = f(c.dc[ch]);
#pragma unroll
        for (int k = 1; k < 16; ++k)
#pragma unroll
            for (int ch = 0; ch < 3; ++ch)
                v[k * 3 + ch] = k - 1 < c.rest_per_ch ? f(c.rest[ch * c.rest_per_ch + k - 1]) : 0.0f;
        float4* dst = reinterpret_cast<float4*>(sh + i * 48);
#pragma unroll
        for (int q = 0; q < 12; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    }
}

bool device_path_ok(const Layout& L, PlyColumns* c) {
    if (!L.binary || L.stride % 4 != 0) return false;
    auto off = [&](int idx) { return L.props[(size_t)idx].offset; };
    int all[14] = {L.pos[0], L.pos[1], L.pos[2], L.scl[0], L.scl[1], L.scl[2], L.rot[0],
                   L.rot[1], L.rot[2], L.rot[3], L.op, L.dc[0], L.dc[1], L.dc[2]};
    for (int k = 0; k < 14; ++k)
        if (off(all[k]) % 4) return false;
    for (int r : L.rest)
        if (off(r) % 4) return false;
    c->stride = L.stride;
    for (int k = 0; k < 3; ++k) { c->pos[k] = off(L.pos[k]); c->scl[k] = off(L.scl[k]); c->dc[k] = off(L.dc[k]); }
    for (int k = 0; k < 4; ++k) c->rot[k] = off(L.rot[k]);
    c->op = off(L.op);
    c->rest_per_ch = L.rest_per_ch;
    for (int k = 0; k < 3 * kMaxRestPerChannel; ++k) c->rest[k] = k < (int)L.rest.size() ? off(L.rest[(size_t)k]) : 0;
    return true;
}

}  // namespace
}  // namespace lumen

using namespace lumen;

extern "C" {

LumenStatus lumen_ply_info(const char* path, int32_t values, LumenPlyInfo* info) {
    if (!path || !info || values < 0 || values > 2) return LUMEN_ERROR_INVALID_ARGUMENT;
    FILE* fp = fopen(path, "rb");
    if (!fp) return LUMEN_ERROR_IO_FAILURE;
    Layout L;
    const LumenStatus st = parse_header(fp, values, &L);
    fclose(fp);
    if (st == LUMEN_SUCCESS) fill_info(L, info);
    return st;
}

LumenStatus lumen_ply_load_host(const char* path, int32_t values, float* means, float* scales, float* quats,
                                float* opacities, float* sh, int64_t capacity, LumenPlyInfo* info) {
    if (!path || values < 0 || values > 2) return LUMEN_ERROR_INVALID_ARGUMENT;
    FILE* fp = fopen(path, "rb");
    if (!fp) return LUMEN_ERROR_IO_FAILURE;
    Layout L;
    LumenStatus st = parse_header(fp, values, &L);
    if (st == LUMEN_SUCCESS && L.count > capacity) st = LUMEN_ERROR_INVALID_ARGUMENT;
    if (st == LUMEN_SUCCESS && L.count > 0 && (!means || !scales || !quats || !opacities || !sh))
        st = LUMEN_ERROR_INVALID_ARGUMENT;
    if (st == LUMEN_SUCCESS) st = load_host(fp, L, means, scales, quats, opacities, sh);
    fclose(fp);
    if (st == LUMEN_SUCCESS) fill_info(L, info);
    return st;
}

LumenStatus lumen_ply_load_device(const char* path, int32_t values, LumenGpuGaussians* dst, LumenPlyInfo* info,
                                  void* stream) {
    if (!path || !dst || values < 0 || values > 2) return LUMEN_ERROR_INVALID_ARGUMENT;
    FILE* fp = fopen(path, "rb");
    if (!fp) return LUMEN_ERROR_IO_FAILURE;
    Layout L;
    LumenStatus st = parse_header(fp, values, &L);
    if (st != LUMEN_SUCCESS) { fclose(fp); return st; }
    if (L.count > dst->count || (L.count > 0 && (!dst->means || !dst->scales || !dst->quats || !dst->opacities ||
                                                 !dst->sh)) ||
        ((uintptr_t)dst->quats & 15u) || ((uintptr_t)dst->sh & 15u)) {
        fclose(fp);
        return LUMEN_ERROR_INVALID_ARGUMENT;
    }
    float* means = const_cast<float*>(dst->means);
    float* scales = const_cast<float*>(dst->scales);
    float* quats = const_cast<float*>(dst->quats);
    float* opac = const_cast<float*>(dst->opacities);
    float* sh = const_cast<float*>(dst->sh);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaSuccess;
    PlyColumns cols;
    if (device_path_ok(L, &cols)) {
        /* two page-locked chunks: read one while the other is copied and de-interleaved */
        const int64_t rows = std::max<int64_t>(1, (int64_t)(64ll << 20) / L.stride);
        const size_t bytes = (size_t)(rows * L.stride);
        unsigned char* host[2] = {nullptr, nullptr};
        unsigned char* dev[2] = {nullptr, nullptr};
        cudaEvent_t done[2] = {nullptr, nullptr};
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            if ((e = cudaHostAlloc(&host[b], bytes, cudaHostAllocDefault)) != cudaSuccess) break;
            if ((e = cudaMalloc(&dev[b], bytes)) != cudaSuccess) break;
            e = cudaEventCreateWithFlags(&done[b], cudaEventDisableTiming);
        }
        int chunk = 0;
        for (int64_t i0 = 0; e == cudaSuccess && st == LUMEN_SUCCESS && i0 < L.count; i0 += rows, ++chunk) {
            const int b = chunk & 1;
            const int64_t nr = L.count - i0 < rows ? L.count - i0 : rows;
            if (chunk >= 2 && (e = cudaEventSynchronize(done[b])) != cudaSuccess) break;
            if (fread(host[b], (size_t)L.stride, (size_t)nr, fp) != (size_t)nr) { st = LUMEN_ERROR_IO_FAILURE; break; }
            if ((e = cudaMemcpyAsync(dev[b], host[b], (size_t)(nr * L.stride), cudaMemcpyHostToDevice, s)) !=
                cudaSuccess)
                break;
            const long long grid = std::min<long long>((nr + 255) / 256, 4096);
            ply_deinterleave_kernel<<<(unsigned int)grid, 256, 0, s>>>(dev[b], nr, i0, cols, means, scales, quats,
                                                                       opac, sh);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
            e = cudaEventRecord(done[b], s);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        for (int b = 0; b < 2; ++b) {
            if (done[b]) cudaEventDestroy(done[b]);
            cudaFree(dev[b]);
            cudaFreeHost(host[b]);
        }
    } else {
        /* parse on the host into page-locked SoA arrays, then upload */
        const size_t n = (size_t)L.count;
        float* hb = nullptr;
        const size_t floats = n * (3 + 3 + 4 + 1 + 48);
        if (n > 0 && (e = cudaHostAlloc(&hb, floats * sizeof(float) + 64, cudaHostAllocDefault)) != cudaSuccess) {
            fclose(fp);
            return map_cuda(e);
        }
        if (n > 0) {
            float* hm = hb;
            float* hs = hm + n * 3;
            float* hq = hs + n * 3;
            float* ho = hq + n * 4;
            float* hsh = ho + n;
            st = load_host(fp, L, hm, hs, hq, ho, hsh);
            if (st == LUMEN_SUCCESS) {
                if ((e = cudaMemcpyAsync(means, hm, n * 3 * sizeof(float), cudaMemcpyHostToDevice, s)) == cudaSuccess &&
                    (e = cudaMemcpyAsync(scales, hs, n * 3 * sizeof(float), cudaMemcpyHostToDevice, s)) == cudaSuccess &&
                    (e = cudaMemcpyAsync(quats, hq, n * 4 * sizeof(float), cudaMemcpyHostToDevice, s)) == cudaSuccess &&
                    (e = cudaMemcpyAsync(opac, ho, n * sizeof(float), cudaMemcpyHostToDevice, s)) == cudaSuccess)
                    e = cudaMemcpyAsync(sh, hsh, n * 48 * sizeof(float), cudaMemcpyHostToDevice, s);
                if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            }
            cudaFreeHost(hb);
        }
    }
    fclose(fp);
    if (e != cudaSuccess) return map_cuda(e);
    if (st != LUMEN_SUCCESS) return st;
    dst->count = L.count;
    fill_info(L, info);
    return LUMEN_SUCCESS;
}

}  // extern "C"
