// Scene I/O: fromPly / toPly (trainer/gpu.js:983-999, :524-531) and toSplat (:538-556),
// with the SH bands >= 1 the reference does not carry (f_rest_*, channel-major as the
// 3DGS .ply convention stores them).
//
// Loading copies the file's body to the device as it is (vertex-major floats) and one
// kernel transposes it into the plane-major parameters, converting f_dc to colour
// (clamp(f_dc SH0 + 0.5, 0, 1) in double, as the reference's JavaScript does); no
// per-Gaussian host objects are built.  Saving runs the inverse kernel and copies the
// body back.  toSplat's 32-byte records (position, scales, colour / opacity / rotation
// bytes) are formed on the device with their sort weights; the host does the stable sort
// by weight, largest first, that the reference does with Array.sort.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace gs {

constexpr double SH0_D = 0.28209479177387814;

// column of each plane in the file (-1: absent -> 0, unit quaternion w for plane 6)
struct PlyMap {
    int col[GS_MAX_PLANES];
    int dc[3];
};

__global__ void ply_to_planes_kernel(const float* __restrict__ body, int nprops, int n, int n_pad, int planes,
                                     PlyMap m, float* __restrict__ params) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad) return;
    const size_t np = (size_t)n_pad;
    if (i >= n) {
        for (int k = 0; k < planes; k++) params[k * np + i] = k == 6 ? 1.f : 0.f;
        return;
    }
    const float* row = body + (size_t)i * nprops;
    for (int k = 0; k < planes; k++) {
        float v = 0.f;
        if (k >= 11 && k <= 13) {
            const double c = (double)row[m.dc[k - 11]] * SH0_D + 0.5;
            v = (float)fmin(1.0, fmax(0.0, c));
            if (isnan(c)) v = __int_as_float(0x7fc00000);  // Math.min/max keep NaN
        } else if (m.col[k] >= 0) {
            v = row[m.col[k]];
        }
        params[k * np + i] = v;
    }
}

__global__ void planes_to_ply_kernel(const float* __restrict__ params, int n, int n_pad, int planes, int nk_out,
                                     int nprops, float* __restrict__ body) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t np = (size_t)n_pad;
    const int nk = (planes - 14) / 3;
    float* row = body + (size_t)i * nprops;
    int o = 0;
    for (int k = 0; k < 3; k++) row[o++] = params[k * np + i];          // x y z
    for (int k = 0; k < 3; k++) row[o++] = 0.f;                         // nx ny nz
    for (int k = 0; k < 3; k++)                                         // f_dc = (c - 0.5) / SH0
        row[o++] = (float)(((double)params[(11 + k) * np + i] - 0.5) / SH0_D);
    for (int c = 0; c < 3; c++)                                         // f_rest, channel-major
        for (int k = 0; k < nk_out; k++) row[o++] = params[(14 + c * nk + k) * np + i];
    row[o++] = params[10 * np + i];                                     // opacity
    for (int k = 0; k < 3; k++) row[o++] = params[(3 + k) * np + i];   // scale_0..2
    for (int k = 0; k < 4; k++) row[o++] = params[(6 + k) * np + i];   // rot_0..3
}

__device__ __forceinline__ unsigned char js_byte(double v) {
    // Math.max(0, Math.min(255, Math.round(v))); Math.round rounds halves up.
    const double r = floor(v + 0.5);
    return (unsigned char)fmin(255.0, fmax(0.0, r));
}

__global__ void splat_records_kernel(const float* __restrict__ params, int n, int n_pad,
                                     unsigned char* __restrict__ rec, double* __restrict__ weight,
                                     unsigned char* __restrict__ finite) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t np = (size_t)n_pad;
    float p[14];
    bool ok = true;
    for (int k = 0; k < 14; k++) {
        p[k] = params[k * np + i];
        ok = ok && isfinite(p[k]);
    }
    finite[i] = ok ? 1 : 0;
    weight[i] = exp((double)p[3] + (double)p[4] + (double)p[5]) / (1.0 + exp(-(double)p[10]));
    float* f = reinterpret_cast<float*>(rec + (size_t)i * 32);
    for (int k = 0; k < 3; k++) f[k] = p[k];
    for (int k = 0; k < 3; k++) f[3 + k] = (float)exp((double)p[3 + k]);
    unsigned char* u = rec + (size_t)i * 32 + 24;
    for (int k = 0; k < 3; k++) u[k] = js_byte((double)p[11 + k] * 255.0);
    u[3] = js_byte(255.0 / (1.0 + exp(-(double)p[10])));
    double len = sqrt((double)p[6] * p[6] + (double)p[7] * p[7] + (double)p[8] * p[8] + (double)p[9] * p[9]);
    if (!(len > 0.0)) len = 1.0;  // Math.hypot(...q) || 1
    for (int k = 0; k < 4; k++) u[4 + k] = js_byte((double)p[6 + k] / len * 128.0 + 128.0);
}

// ---- host ------------------------------------------------------------------------------
int ply_parse(const void* data, int64_t bytes, int planes, PlyHeaderInfo* out, std::string* err) {
    const char* s = static_cast<const char*>(data);
    // The reference looks for the header in the first 4096 bytes.
    const int64_t scan = std::min<int64_t>(bytes, 4096);
    const std::string head(s, (size_t)scan);
    const size_t e = head.find("end_header\n");
    if (e == std::string::npos) {
        *err = "no end_header in the first 4096 bytes";
        return -1;
    }
    out->header_bytes = (int64_t)(e + strlen("end_header\n"));
    const std::string header = head.substr(0, (size_t)out->header_bytes);
    if (header.compare(0, 4, "ply\n") != 0 || header.find("format binary_little_endian 1.0") == std::string::npos) {
        *err = "not a binary little-endian .ply";
        return -1;
    }
    const size_t v = header.find("element vertex ");
    if (v == std::string::npos) {
        *err = "no vertex element";
        return -1;
    }
    out->count = atoll(header.c_str() + v + strlen("element vertex "));
    std::vector<std::string> props;
    size_t pos = 0;
    while ((pos = header.find("property ", pos)) != std::string::npos) {
        const size_t eol = header.find('\n', pos);
        const std::string line = header.substr(pos, eol - pos);
        pos = eol;
        char type[32] = {0}, name[128] = {0};
        if (sscanf(line.c_str(), "property %31s %127s", type, name) != 2 || strcmp(type, "float") != 0) {
            *err = "only float vertex properties are read: " + line;
            return -1;
        }
        props.push_back(name);
    }
    out->nprops = (int)props.size();
    if (out->count < 0 || out->header_bytes + out->count * out->nprops * 4 > bytes) {
        *err = "file shorter than its header says";
        return -1;
    }
    auto find = [&](const std::string& n) -> int {
        for (size_t k = 0; k < props.size(); k++)
            if (props[k] == n) return (int)k;
        return -1;
    };
    const char* need[] = {"x", "y", "z", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3",
                          "opacity", "f_dc_0", "f_dc_1", "f_dc_2"};
    const int plane_of[] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13};
    for (int k = 0; k < GS_MAX_PLANES; k++) out->col[k] = -1;
    for (int k = 0; k < 14; k++) {
        const int c = find(need[k]);
        if (c < 0) {
            *err = std::string("missing property ") + need[k];
            return -1;
        }
        out->col[plane_of[k]] = c;
    }
    for (int k = 0; k < 3; k++) out->dc[k] = out->col[11 + k];
    // f_rest: channel-major with rest/3 coefficients per channel in the file.
    int rest = 0;
    while (find("f_rest_" + std::to_string(rest)) >= 0) rest++;
    out->file_sh_coeffs = rest / 3;
    const int nk = (planes - 14) / 3;
    for (int c = 0; c < 3; c++)
        for (int k = 0; k < nk && k < out->file_sh_coeffs; k++)
            out->col[14 + c * nk + k] = find("f_rest_" + std::to_string(c * out->file_sh_coeffs + k));
    return 0;
}

void launch_ply_to_planes(const float* body, const PlyHeaderInfo& h, int n_pad, int planes, float* params,
                          cudaStream_t s) {
    PlyMap m;
    for (int k = 0; k < GS_MAX_PLANES; k++) m.col[k] = h.col[k];
    for (int k = 0; k < 3; k++) m.dc[k] = h.dc[k];
    const int blocks = (n_pad + 255) / 256;
    if (blocks > 0) ply_to_planes_kernel<<<blocks, 256, 0, s>>>(body, h.nprops, (int)h.count, n_pad, planes, m, params);
}

std::string ply_header(int64_t n, int nk_out) {
    std::string h = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(n) + "\n";
    const char* a[] = {"x", "y", "z", "nx", "ny", "nz", "f_dc_0", "f_dc_1", "f_dc_2"};
    for (const char* p : a) h += std::string("property float ") + p + "\n";
    for (int k = 0; k < 3 * nk_out; k++) h += "property float f_rest_" + std::to_string(k) + "\n";
    const char* b[] = {"opacity", "scale_0", "scale_1", "scale_2", "rot_0", "rot_1", "rot_2", "rot_3"};
    for (const char* p : b) h += std::string("property float ") + p + "\n";
    h += "end_header\n";
    return h;
}

void launch_planes_to_ply(const float* params, int n, int n_pad, int planes, int nk_out, float* body,
                          cudaStream_t s) {
    const int nprops = 17 + 3 * nk_out;
    if (n > 0) planes_to_ply_kernel<<<(n + 255) / 256, 256, 0, s>>>(params, n, n_pad, planes, nk_out, nprops, body);
}

void launch_splat_records(const float* params, int n, int n_pad, unsigned char* rec, double* weight,
                          unsigned char* finite, cudaStream_t s) {
    if (n > 0) splat_records_kernel<<<(n + 255) / 256, 256, 0, s>>>(params, n, n_pad, rec, weight, finite);
}

// Order of toSplat: finite Gaussians by weight, largest first, ties in index order.
std::vector<int> splat_order(const std::vector<double>& weight, const std::vector<unsigned char>& finite) {
    std::vector<int> idx;
    idx.reserve(weight.size());
    for (size_t i = 0; i < weight.size(); i++)
        if (finite[i]) idx.push_back((int)i);
    // Array.sort with (a, b) => b[0] - a[0]: NaN comparisons count as equal.
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return weight[(size_t)b] - weight[(size_t)a] < 0; });
    return idx;
}

}  // namespace gs
