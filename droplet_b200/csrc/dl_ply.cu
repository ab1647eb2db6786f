// dl_ply.cu — 3DGS PLY loading behind the C ABI (src/io/ply.ts:41-239).
//
// Parses a binary little-endian PLY held in memory straight into the SoA
// arrays of dl_splats (optionally page-locked, so that dl_scene_upload /
// dl_render copy them to the device at full PCIe rate with no staging copy).
// Accepted layouts, transforms and error messages are the reference loader's:
//   * header: the first 64 KB must contain "end_header\n"; lines trimmed,
//     empty lines dropped; "ply" magic; "format" with "binary" and
//     "little_endian"; the `vertex` element's properties of type float, uchar
//     or int (other elements end the vertex section); count > 0;
//   * every vertex property float; fields found by name (a repeated name
//     keeps its last position), in the reference's order of checks;
//   * positions with y negated when flipY; log-scales and opacity logits as
//     stored; f_dc_* times SH_C0 = 1/(2 sqrt(pi)) in double, rounded once to
//     float; quaternion (rot_0..3 = w, x, y, z) divided by its norm in
//     double (Math.hypot(...) || 1: NaN and 0 norms divide by 1, an infinite
//     component gives an infinite norm), x and z negated when flipY;
//   * f_rest_0.. (consecutive names) give coeffsPerChannel = floor(k / 3) and
//     the SH band; the coefficients are copied per splat in f_rest order.
// Two deliberate differences, shared with the Python loader
// (droplet_b200/ply.py): an f_rest count whose coeffsPerChannel is none of
// 3, 8, 15 is an error (the reference would return an SH stride that
// disagrees with its shBands), and an `element vertex` line without digits is
// "no vertices" (the reference's parseInt gives NaN and an empty result).
// The norm is the square root of the double sum of squares (Math.hypot may
// differ in the last double ulp, below the float rounding that follows).
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <string>
#include <unordered_map>
#include <vector>

#include "dl_internal.h"

struct dl_ply {
    uint64_t count = 0;
    int sh_bands = 0;
    uint32_t sh_stride = 0;        // floats of SH per splat (3 * coeffsPerChannel)
    bool pinned = false;
    float* block = nullptr;        // one allocation: positions | rotations | logScales | opacity | dc | sh
    float *pos = nullptr, *rot = nullptr, *lsc = nullptr, *opl = nullptr, *dc = nullptr, *sh = nullptr;
};

namespace {

constexpr double kShC0 = 0.28209479177387814;   // ply.ts:23
constexpr size_t kHeaderMax = 65536;            // ply.ts:45

std::string trim(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && (unsigned char)s[a] <= ' ') a++;
    while (b > a && (unsigned char)s[b - 1] <= ' ') b--;
    return s.substr(a, b - a);
}

bool starts(const std::string& s, const char* p) { return s.compare(0, std::strlen(p), p) == 0; }

struct Prop { std::string type, name; };

int fail(const std::string& msg) {
    dl_set_error(msg);
    return DL_E_INVALID_ARG;
}

// ply.ts:41-92
int parse_header(const uint8_t* bytes, size_t len, int64_t* count, std::vector<Prop>* props, size_t* offset) {
    const size_t n = len < kHeaderMax ? len : kHeaderMax;
    const std::string head(reinterpret_cast<const char*>(bytes), n);
    const size_t end = head.find("end_header\n");
    if (end == std::string::npos) return fail("PLY: end_header not found in first 64KB");
    *offset = end + std::strlen("end_header\n");
    std::vector<std::string> lines;
    size_t p = 0;
    while (p <= end) {
        size_t q = head.find('\n', p);
        if (q == std::string::npos || q > end) q = end;
        const std::string l = trim(head.substr(p, q - p));
        if (!l.empty()) lines.push_back(l);
        p = q + 1;
    }
    if (lines.empty() || lines[0] != "ply") return fail("PLY: missing magic");
    bool binary = false, little = true, inVertex = false;
    *count = 0;
    for (size_t i = 1; i < lines.size(); i++) {
        const std::string& line = lines[i];
        if (starts(line, "format ")) {
            binary = line.find("binary") != std::string::npos;
            little = line.find("little_endian") != std::string::npos;
            continue;
        }
        if (starts(line, "element vertex ")) {
            // parseInt(.., 10): leading white space, a sign, then digits
            const char* s = line.c_str() + std::strlen("element vertex ");
            while (*s == ' ' || *s == '\t') s++;
            const char* d = s + ((*s == '+' || *s == '-') ? 1 : 0);
            if (*d >= '0' && *d <= '9') {
                const long long v = std::strtoll(s, nullptr, 10);
                *count = v;
            } else {
                *count = -1;
            }
            inVertex = true;
            continue;
        }
        if (starts(line, "element ")) {
            inVertex = false;
            continue;
        }
        if (inVertex && starts(line, "property ")) {
            std::vector<std::string> parts;
            size_t a = 0;
            while (a < line.size()) {
                while (a < line.size() && (unsigned char)line[a] <= ' ') a++;
                size_t b = a;
                while (b < line.size() && (unsigned char)line[b] > ' ') b++;
                if (b > a) parts.push_back(line.substr(a, b - a));
                a = b;
            }
            const std::string t = parts.size() > 1 ? parts[1] : "";
            const std::string name = parts.size() > 2 ? parts[2] : "";
            if (t != "float" && t != "uchar" && t != "int") return fail("PLY: unsupported property type \"" + t + "\"");
            props->push_back({t, name});
        }
    }
    if (!binary) return fail("PLY: ASCII PLY not supported (binary only)");
    if (!little) return fail("PLY: only little-endian supported");
    if (*count <= 0) return fail("PLY: no vertices");
    return DL_OK;
}

void release(dl_ply* p) {
    if (!p || !p->block) return;
    if (p->pinned) cudaFreeHost(p->block);
    else std::free(p->block);
    p->block = nullptr;
}

}  // namespace

extern "C" int dl_ply_load(const uint8_t* bytes, size_t len, int flip_y, uint32_t flags, dl_ply** out) {
    if (!out) return fail("dl_ply_load: NULL argument");
    *out = nullptr;
    if (!bytes && len) return fail("dl_ply_load: NULL bytes");
    int64_t count = 0;
    std::vector<Prop> props;
    size_t offset = 0;
    DL_TRY(parse_header(bytes, len, &count, &props, &offset));

    // ply.ts:130-165
    std::unordered_map<std::string, size_t> idx;
    for (size_t p = 0; p < props.size(); p++) idx[props[p].name] = p;
    for (const Prop& p : props)
        if (p.type != "float") return fail("PLY: mixed property types not yet supported");
    const uint64_t per = props.size();
    const uint64_t total = (uint64_t)count * per * 4;
    if (offset + total > len)
        return fail("PLY: data section truncated (need " + std::to_string(total) + " bytes, have " +
                    std::to_string(len - offset) + ")");
    const char* names[] = {"x", "y", "z", "scale_0", "scale_1", "scale_2", "f_dc_0", "f_dc_1", "f_dc_2",
                           "opacity", "rot_0", "rot_1", "rot_2", "rot_3"};
    size_t ix[14];
    for (int k = 0; k < 14; k++) {
        auto it = idx.find(names[k]);
        if (it == idx.end()) return fail(std::string("PLY: missing property \"") + names[k] + "\"");
        ix[k] = it->second;
    }
    // ply.ts:172-180: consecutive f_rest_k
    std::vector<size_t> rest;
    while (true) {
        auto it = idx.find("f_rest_" + std::to_string(rest.size()));
        if (it == idx.end()) break;
        rest.push_back(it->second);
    }
    const uint32_t cpc = (uint32_t)(rest.size() / 3);
    const int bands = cpc >= 15 ? 3 : cpc >= 8 ? 2 : cpc >= 3 ? 1 : 0;
    if (bands && cpc != (bands == 1 ? 3u : bands == 2 ? 8u : 15u))
        return fail("PLY: " + std::to_string(rest.size()) + " f_rest properties match no SH band layout (9, 24 or 45)");

    dl_ply* P = new dl_ply();
    P->count = (uint64_t)count;
    P->sh_bands = bands;
    P->sh_stride = bands ? 3 * cpc : 0;
    const uint64_t N = P->count;
    const uint64_t floats = N * (3 + 4 + 3 + 1 + 3 + (uint64_t)P->sh_stride);
    P->pinned = (flags & DL_PLY_PINNED) != 0;
    if (P->pinned) {
        const cudaError_t e = cudaHostAlloc((void**)&P->block, floats * 4, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            P->block = nullptr;
            delete P;
            dl_set_error(std::string("dl_ply_load: cudaHostAlloc: ") + cudaGetErrorString(e));
            return e == cudaErrorMemoryAllocation ? DL_E_OOM : DL_E_CUDA;
        }
    } else {
        P->block = static_cast<float*>(std::malloc(floats * 4));
        if (!P->block) {
            delete P;
            dl_set_error("dl_ply_load: out of host memory");
            return DL_E_OOM;
        }
    }
    P->pos = P->block;
    P->rot = P->pos + 3 * N;
    P->lsc = P->rot + 4 * N;
    P->opl = P->lsc + 3 * N;
    P->dc = P->opl + N;
    P->sh = bands ? P->dc + 3 * N : nullptr;

    // ply.ts:192-235 (the data need not be 4-byte aligned: read through memcpy)
    const uint8_t* data = bytes + offset;
    const double ySign = flip_y ? -1.0 : 1.0;
    std::vector<float> row(per);
    for (uint64_t i = 0; i < N; i++) {
        std::memcpy(row.data(), data + i * per * 4, per * 4);
        P->pos[i * 3 + 0] = row[ix[0]];
        P->pos[i * 3 + 1] = (float)(ySign * (double)row[ix[1]]);
        P->pos[i * 3 + 2] = row[ix[2]];
        P->lsc[i * 3 + 0] = row[ix[3]];
        P->lsc[i * 3 + 1] = row[ix[4]];
        P->lsc[i * 3 + 2] = row[ix[5]];
        P->opl[i] = row[ix[9]];
        P->dc[i * 3 + 0] = (float)(kShC0 * (double)row[ix[6]]);
        P->dc[i * 3 + 1] = (float)(kShC0 * (double)row[ix[7]]);
        P->dc[i * 3 + 2] = (float)(kShC0 * (double)row[ix[8]]);
        const double w = row[ix[10]], qx = row[ix[11]], qy = row[ix[12]], qz = row[ix[13]];
        double n = std::sqrt(((w * w + qx * qx) + qy * qy) + qz * qz);
        if (std::isinf(w) || std::isinf(qx) || std::isinf(qy) || std::isinf(qz)) n = INFINITY;
        if (std::isnan(n) || n == 0.0) n = 1.0;                      // Math.hypot(...) || 1
        const double f = flip_y ? -1.0 : 1.0;
        P->rot[i * 4 + 0] = (float)(w / n);
        P->rot[i * 4 + 1] = (float)((f * qx) / n);
        P->rot[i * 4 + 2] = (float)(qy / n);
        P->rot[i * 4 + 3] = (float)((f * qz) / n);
        for (uint32_t k = 0; k < P->sh_stride; k++) P->sh[i * P->sh_stride + k] = row[rest[k]];
    }
    *out = P;
    return DL_OK;
}

extern "C" int dl_ply_splats(const dl_ply* p, dl_splats* out) {
    if (!p || !out) return fail("dl_ply_splats: NULL argument");
    out->count = p->count;
    out->positions = p->pos;
    out->rotations = p->rot;
    out->log_scales = p->lsc;
    out->opacity_logits = p->opl;
    out->colors_dc = p->dc;
    out->colors_sh = p->sh;
    out->sh_bands = p->sh_bands;
    return DL_OK;
}

extern "C" int dl_ply_free(dl_ply* p) {
    if (!p) return DL_OK;
    release(p);
    delete p;
    return DL_OK;
}
