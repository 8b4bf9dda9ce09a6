// io.cpp -- scene input, ray files and image output (host side, no GPU).
//
// Reference formats (javorkk/happyray):
//   scene.cfg      src/Application/SceneConfigurationReader.cpp:29-190
//   frame names    src/Application/AnimationLoader.cpp:50-101
//   OBJ            src/Application/WFObjectReader.cpp:320-560
//   camera.cfg     src/Application/CameraManager.cpp:33-168
//   light.cfg      src/Application/LightSourceLoader.cpp:29-110
//   .rays          src/RT/Integrator/SimpleRayTraverser.h:200-261
//   PNG            src/Utils/ImagePNG.cpp:160-215
// The OBJ reader parses line chunks of the file in parallel (the reference parses one
// line at a time): each chunk collects its vertices and raw face indices, the chunks'
// vertex counts give every chunk's first global vertex, and relative (negative) indices
// are resolved against them.  The PNG writer emits stored (uncompressed) deflate blocks
// with its own CRC-32 and Adler-32, so it needs no compression library.
#include "../../include/happyray.h"

#include <cstdint>
#include <functional>

#include <algorithm>
#include <cerrno>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <new>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

struct hr_scene {
    std::vector<float> kf;          // K x V x 3
    std::vector<uint32_t> idx;      // N x 3
    uint32_t nv = 0, nt = 0, nkf = 0;
    float frame_step = 0.0f;
    bool has_camera = false;
    float pos[3] = {0, 0, 0}, orient[3] = {0, 0, -1}, up[3] = {0, 1, 0};
    float fov = 60.0f;
    int32_t w = 0, h = 0;
    struct QuadLight { float position[3], normal[3], intensity[3], edge1[3], edge2[3]; };
    std::vector<QuadLight> lights;
    std::vector<float> normals;     // shading normals, M x 3 (empty: the file had none)
    std::vector<uint32_t> nidx;     // N x 3 normal indices, with normals
    std::vector<float> albedo;      // material table (empty: no usemtl / mtllib)
    std::vector<uint32_t> tri_mat;  // N material indices, with albedo
};

namespace {

thread_local std::string g_err;

hr_status io_error(hr_status code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

bool read_file(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    f.seekg(0, std::ios::end);
    const std::streamoff n = f.tellg();
    if (n < 0) return false;
    out.resize((size_t)n);
    f.seekg(0, std::ios::beg);
    if (n > 0) f.read(&out[0], n);
    return (bool)f;
}

// ---------------------------------------------------------------------------------
// OBJ

struct ObjChunk {
    std::vector<float> v;
    std::vector<int64_t> face;       // triangle corners: > 0 global 1-based, < 0 relative
    std::vector<uint32_t> face_vcount;   // local vertex count when the corner was read
    std::vector<float> n;            // vn triples
    // normal index per triangle corner (0: none, else as `face`), kept only once a corner
    // of this chunk named one; shorter than `face` means "none" for the corners past it
    std::vector<int64_t> fnorm;
    std::vector<uint32_t> face_ncount;   // local normal count when the corner was read
    std::vector<std::pair<size_t, std::string>> usemtl;   // (triangles before it, name)
    std::vector<std::string> mtllib;
    size_t first_line = 0;
    std::string err;
};

// what an OBJ file holds besides positions and triangles
struct ObjExtras {
    std::vector<float> normals;          // the file's vn, then one geometric normal per face lacking one
    std::vector<uint32_t> nidx;          // 3 per triangle; empty when the file has no vn
    std::vector<std::string> mat_names;  // "Default" first, then in order of first usemtl
    std::vector<float> albedo;           // per material
    std::vector<uint32_t> tri_mat;       // per triangle; empty when the file names no material
};

inline bool starts_with_ci(const char* s, const char* e, const char* w) {
    for (; *w; ++w, ++s)
        if (s >= e || std::tolower((unsigned char)*s) != *w) return false;
    return true;
}

std::string trimmed(const char* s, const char* e) {
    while (s < e && (*s == ' ' || *s == '\t')) ++s;
    while (e > s && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\r')) --e;
    return std::string(s, e);
}

inline const char* skip_ws(const char* s, const char* e) {
    while (s < e && (*s == ' ' || *s == '\t' || *s == '\r')) ++s;
    return s;
}

// one line of an OBJ file; returns false with c.err set on a malformed line
bool obj_line(const char* s, const char* e, ObjChunk& c, size_t line) {
    s = skip_ws(s, e);
    // comments end the line
    const char* hash = (const char*)std::memchr(s, '#', (size_t)(e - s));
    if (hash) e = hash;
    while (e > s && (e[-1] == ' ' || e[-1] == '\t' || e[-1] == '\r')) --e;
    if (s >= e) return true;
    const char k = (char)std::tolower((unsigned char)s[0]);
    if (k == 'v') {
        const bool is_n = s + 2 < e && (s[1] == 'n' || s[1] == 'N') && (s[2] == ' ' || s[2] == '\t');
        if ((s + 1 < e && (s[1] == ' ' || s[1] == '\t')) || is_n) {
            // position or normal: exactly three numbers (WFObjectReader.cpp:354-386)
            const char* p = s + (is_n ? 2 : 1);
            float xyz[3];
            int n = 0;
            std::string tmp(p, e);
            const char* q = tmp.c_str();
            for (;;) {
                while (*q == ' ' || *q == '\t') ++q;
                if (!*q) break;
                char* end;
                const double d = std::strtod(q, &end);
                if (end == q || n >= 3) {
                    c.err = "line " + std::to_string(line) + ": a vertex needs three numbers";
                    return false;
                }
                xyz[n++] = (float)d;
                q = end;
            }
            if (n != 3) {
                c.err = "line " + std::to_string(line) + ": a vertex needs three numbers";
                return false;
            }
            (is_n ? c.n : c.v).insert((is_n ? c.n : c.v).end(), xyz, xyz + 3);
        }
        return true;   // vt: not needed by the hot path
    }
    // 'f' (or "fo") and, as in the reference, 'l': three or more corners make triangles
    if ((k == 'f' || k == 'l') && s + 1 < e && (s[1] == ' ' || s[1] == '\t' || s[1] == 'o' || s[1] == 'O')) {
        std::string tmp(s + (s[1] == 'o' || s[1] == 'O' ? 2 : 1), e);
        const char* q = tmp.c_str();
        std::vector<int64_t> poly, pnorm;
        bool any_n = false;
        for (;;) {
            while (*q == ' ' || *q == '\t') ++q;
            if (!*q) break;
            char* end;
            const long long vi = std::strtoll(q, &end, 10);
            if (end == q || vi == 0) {
                c.err = "line " + std::to_string(line) + ": bad face index";
                return false;
            }
            q = end;
            // v, v/t, v//n or v/t/n (WFObjectReader.cpp:411-470): the texture index is skipped
            long long ni = 0;
            if (*q == '/') {
                ++q;
                if (*q != '/') {
                    std::strtoll(q, &end, 10);
                    if (end == q) {
                        c.err = "line " + std::to_string(line) + ": bad face index";
                        return false;
                    }
                    q = end;
                }
                if (*q == '/') {
                    ++q;
                    ni = std::strtoll(q, &end, 10);
                    if (end == q || ni == 0) {
                        c.err = "line " + std::to_string(line) + ": bad normal index";
                        return false;
                    }
                    q = end;
                }
            }
            poly.push_back(vi);
            pnorm.push_back(ni);
            any_n |= ni != 0;
        }
        if (poly.size() < 3) return true;   // points and lines are not triangles
        const uint32_t vc = (uint32_t)(c.v.size() / 3), ncnt = (uint32_t)(c.n.size() / 3);
        if (any_n) {   // align the normal-index arrays with the corners before this face
            c.fnorm.resize(c.face.size(), 0);
            c.face_ncount.resize(c.face.size(), 0);
        }
        for (size_t i = 1; i + 1 < poly.size(); ++i) {   // fan from the first corner
            const size_t cs[3] = {0, i, i + 1};
            for (int t = 0; t < 3; ++t) {
                c.face.push_back(poly[cs[t]]);
                c.face_vcount.push_back(vc);
                if (any_n) {
                    c.fnorm.push_back(pnorm[cs[t]]);
                    c.face_ncount.push_back(ncnt);
                }
            }
        }
        return true;
    }
    // materials (WFObjectReader.cpp:541-565): usemtl selects one for the faces after it,
    // mtllib names a .mtl file read once the OBJ is parsed
    if (starts_with_ci(s, e, "usemtl") && s + 6 < e && (s[6] == ' ' || s[6] == '\t')) {
        const std::string name = trimmed(s + 6, e);
        if (!name.empty()) c.usemtl.emplace_back(c.face.size() / 3, name);
        return true;
    }
    if (starts_with_ci(s, e, "mtllib") && s + 6 < e && (s[6] == ' ' || s[6] == '\t')) {
        const std::string name = trimmed(s + 6, e);
        if (!name.empty()) c.mtllib.push_back(name);
        return true;
    }
    return true;   // o, g, s, p and anything else: skipped
}

// A .mtl file (readMtlLib, WFObjectReader.cpp:135-258): "newmtl name" selects a material the
// OBJ named (an unknown name leaves the selection as it was, as the reference does), "Kd r g
// b" sets its diffuse colour.  The path tracer's albedo is the grey of the reference's
// normalised reflectance (setupPhongCoefficients, WFObjectReader.cpp:49-57: min(Kd, 0.99)
// per channel; the 1/pi of its BRDF is applied by the tracer): the mean of the three.
hr_status read_mtl(const std::string& path, const std::vector<std::string>& names, std::vector<float>& albedo) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return io_error(HR_ERR_INVALID_ARG, "cannot read .mtl file %s", path.c_str());
    std::string line;
    long cur = -1;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        const char* s = skip_ws(line.data(), line.data() + line.size());
        const char* e = line.data() + line.size();
        if (starts_with_ci(s, e, "newmtl")) {
            const std::string name = trimmed(s + 6, e);
            const auto it = std::find(names.begin(), names.end(), name);
            if (it != names.end()) cur = (long)(it - names.begin());
        } else if (starts_with_ci(s, e, "kd") && cur >= 0) {
            std::string tmp(s + 2, e);
            const char* q = tmp.c_str();
            float kd[3];
            int n = 0;
            for (; n < 3; ++n) {
                char* end;
                kd[n] = std::strtof(q, &end);
                if (end == q) break;
                q = end;
            }
            if (n == 3)
                albedo[(size_t)cur] = (std::min(kd[0], 0.99f) + std::min(kd[1], 0.99f) + std::min(kd[2], 0.99f)) / 3.0f;
        }
    }
    return HR_OK;
}

void obj_parse_chunk(const char* b, const char* e, ObjChunk& c) {
    size_t line = c.first_line;
    while (b < e) {
        const char* nl = (const char*)std::memchr(b, '\n', (size_t)(e - b));
        const char* le = nl ? nl : e;
        ++line;
        if (!obj_line(b, le, c, line)) return;
        b = nl ? nl + 1 : e;
    }
}

std::string dir_of(const std::string& p);

constexpr uint32_t kNoNormal = 0xffffffffu;

// every triangle with a corner lacking a normal index gets one appended normal, its
// normalised edge1 x edge2, for those corners (WFObjectReader.cpp:602-614)
bool fill_geometric_normals(std::vector<float>& normals, std::vector<uint32_t>& nidx, const float* v,
                            const std::vector<uint32_t>& idx) {
    const size_t nt = idx.size() / 3;
    for (size_t t = 0; t < nt; ++t) {
        uint32_t* ni = &nidx[3 * t];
        if (ni[0] != kNoNormal && ni[1] != kNoNormal && ni[2] != kNoNormal) continue;
        const float* a = &v[3 * (size_t)idx[3 * t]];
        const float* b = &v[3 * (size_t)idx[3 * t + 1]];
        const float* d = &v[3 * (size_t)idx[3 * t + 2]];
        const float e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
        const float e2[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
        float n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        const float len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
        for (int k = 0; k < 3; ++k) n[k] = len > 0.0f ? n[k] / len : 0.0f;
        const size_t at = normals.size() / 3;
        if (at >= kNoNormal) return false;
        normals.insert(normals.end(), n, n + 3);
        for (int k = 0; k < 3; ++k)
            if (ni[k] == kNoNormal) ni[k] = (uint32_t)at;
    }
    return true;
}

// Normals and materials of a parsed OBJ (WFObjectReader.cpp:583-640).  With any vn in the
// file, every face lacking a normal index at some corner gets one appended geometric normal
// (normalised edge1 x edge2 of its vertices) for those corners; a file without vn keeps no
// normals (the tracer's geometric normal).  Materials: "Default" (diffuse 0.6774,
// WFObjectReader.cpp:277-283) at index 0, then each usemtl name in order of first use; the
// file's mtllib files, relative to its directory, fill in their Kd.
hr_status obj_extras(const std::string& path, const std::vector<ObjChunk>& ch, const std::vector<float>& v,
                     const std::vector<uint32_t>& idx, ObjExtras& ex) {
    ex = ObjExtras();
    const size_t nt = idx.size() / 3;
    size_t nn = 0;
    for (const auto& c : ch) nn += c.n.size() / 3;
    if (nn > 0xffffffffull) return io_error(HR_ERR_INVALID_ARG, "%s: too many normals", path.c_str());
    if (nn > 0) {
        ex.normals.reserve(3 * nn);
        ex.nidx.assign(3 * nt, kNoNormal);
        uint64_t noff = 0;
        size_t corner = 0;
        for (const auto& c : ch) {
            ex.normals.insert(ex.normals.end(), c.n.begin(), c.n.end());
            for (size_t i = 0; i < c.fnorm.size(); ++i) {
                const int64_t f = c.fnorm[i];
                if (f == 0) continue;
                const int64_t g = f > 0 ? f - 1 : (int64_t)(noff + c.face_ncount[i]) + f;
                if (g < 0 || (uint64_t)g >= nn)
                    return io_error(HR_ERR_INVALID_ARG, "%s: normal index %lld out of range of %zu normals",
                                    path.c_str(), (long long)f, nn);
                ex.nidx[corner + i] = (uint32_t)g;
            }
            corner += c.face.size();
            noff += c.n.size() / 3;
        }
        if (!fill_geometric_normals(ex.normals, ex.nidx, v.data(), idx))
            return io_error(HR_ERR_INVALID_ARG, "%s: too many normals", path.c_str());
    }
    bool any_mat = false;
    for (const auto& c : ch) any_mat |= !c.usemtl.empty() || !c.mtllib.empty();
    if (!any_mat) return HR_OK;
    ex.mat_names.push_back("Default");
    ex.albedo.push_back(0.6774f);
    ex.tri_mat.assign(nt, 0);
    uint32_t cur = 0;
    size_t tri0 = 0;
    for (const auto& c : ch) {
        const size_t ntc = c.face.size() / 3;
        size_t at = 0;
        for (size_t u = 0; u <= c.usemtl.size(); ++u) {
            const size_t upto = u < c.usemtl.size() ? c.usemtl[u].first : ntc;
            std::fill(ex.tri_mat.begin() + (tri0 + at), ex.tri_mat.begin() + (tri0 + upto), cur);
            at = upto;
            if (u == c.usemtl.size()) break;
            const std::string& name = c.usemtl[u].second;
            const auto it = std::find(ex.mat_names.begin(), ex.mat_names.end(), name);
            if (it != ex.mat_names.end()) {
                cur = (uint32_t)(it - ex.mat_names.begin());
            } else {   // a new material: the reference's Material(name) has diffuse 0
                cur = (uint32_t)ex.mat_names.size();
                ex.mat_names.push_back(name);
                ex.albedo.push_back(0.0f);
            }
        }
        tri0 += ntc;
    }
    const std::string dir = dir_of(path);
    for (const auto& c : ch)
        for (const auto& lib : c.mtllib) {
            const hr_status st = read_mtl(lib[0] == '/' ? lib : dir + lib, ex.mat_names, ex.albedo);
            if (st != HR_OK) return st;
        }
    return HR_OK;
}

hr_status read_obj(const std::string& path, int threads, std::vector<float>& v, std::vector<uint32_t>& idx,
                   ObjExtras* ex = nullptr) {
    std::string text;
    if (!read_file(path, text)) return io_error(HR_ERR_INVALID_ARG, "cannot read %s", path.c_str());
    if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
    const size_t n = text.size();
    const int nc = (int)std::max<size_t>(1, std::min<size_t>((size_t)threads, n / (1u << 20) + 1));
    std::vector<size_t> cut(nc + 1, 0);
    cut[nc] = n;
    for (int i = 1; i < nc; ++i) {   // chunk boundaries just after a newline
        size_t p = std::max(cut[i - 1], n * (size_t)i / (size_t)nc);
        while (p < n && text[p - 1] != '\n') ++p;
        cut[i] = p;
    }
    std::vector<ObjChunk> ch(nc);
    for (int i = 0; i < nc; ++i)   // line numbers for messages
        ch[i].first_line = i == 0 ? 0 : ch[i - 1].first_line +
                                            (size_t)std::count(text.begin() + cut[i - 1], text.begin() + cut[i], '\n');
    std::vector<std::thread> th;
    for (int i = 1; i < nc; ++i)
        th.emplace_back(obj_parse_chunk, text.data() + cut[i], text.data() + cut[i + 1], std::ref(ch[i]));
    obj_parse_chunk(text.data() + cut[0], text.data() + cut[1], ch[0]);
    for (auto& t : th) t.join();
    size_t nv = 0, nf = 0;
    for (auto& c : ch) {
        if (!c.err.empty()) return io_error(HR_ERR_INVALID_ARG, "%s: %s", path.c_str(), c.err.c_str());
        nv += c.v.size() / 3;
        nf += c.face.size();
    }
    if (nv > 0xffffffffull || nf / 3 > 0xffffffffull) return io_error(HR_ERR_INVALID_ARG, "%s: too large", path.c_str());
    v.clear();
    v.reserve(nv * 3);
    idx.clear();
    idx.reserve(nf);
    uint64_t voff = 0;
    for (auto& c : ch) {
        v.insert(v.end(), c.v.begin(), c.v.end());
        for (size_t i = 0; i < c.face.size(); ++i) {
            const int64_t f = c.face[i];
            // 1-based global, or relative to the vertices read before this line
            const int64_t g = f > 0 ? f - 1 : (int64_t)(voff + c.face_vcount[i]) + f;
            if (g < 0 || (uint64_t)g >= nv)
                return io_error(HR_ERR_INVALID_ARG, "%s: face index %lld out of range of %zu vertices", path.c_str(),
                                (long long)f, nv);
            idx.push_back((uint32_t)g);
        }
        voff += c.v.size() / 3;
    }
    return ex ? obj_extras(path, ch, v, idx, *ex) : HR_OK;
}

// ---------------------------------------------------------------------------------
// configuration files

std::string trim(const std::string& s) {
    const size_t b = s.find_first_not_of(" \t\r");
    if (b == std::string::npos) return "";
    const size_t e = s.find_last_not_of(" \t\r");
    return s.substr(b, e - b + 1);
}

std::string dir_of(const std::string& p) {
    const size_t s = p.find_last_of('/');
    return s == std::string::npos ? std::string() : p.substr(0, s + 1);
}

std::string resolve(const std::string& p, const std::string& base_dir) {
    std::ifstream f(p);
    if (f || p.empty() || p[0] == '/' || base_dir.empty()) return p;
    return base_dir + p;
}

bool file_exists(const std::string& p) { return (bool)std::ifstream(p); }

// CameraManager::rotate (CameraManager.cpp:33-66): Euler angles in degrees applied to
// the orientation and up vectors
void camera_rotate(float* o, float* u, const float* r) {
    const float ax = r[0] * 3.14159265358979323846f / 180.0f;
    const float ay = r[1] * 3.14159265358979323846f / 180.0f;
    const float az = r[2] * 3.14159265358979323846f / 180.0f;
    const float sx = std::sin(ax), cx = std::cos(ax), sy = std::sin(ay), cy = std::cos(ay), sz = std::sin(az),
                cz = std::cos(az);
    const float c1[3] = {cy * cz, sx * sy * cz - cx * sz, cx * sy * cz + sx * sz};
    const float c2[3] = {cy * sz, sx * sy * sz + cx * cz, sx * sy * sz - sx * cz};
    const float c3[3] = {-sy, sx * cy, cx * cy};
    float no[3], nu[3];
    for (int k = 0; k < 3; ++k) {
        no[k] = c1[k] * o[0] + c2[k] * o[1] + c3[k] * o[2];
        nu[k] = c1[k] * u[0] + c2[k] * u[1] + c3[k] * u[2];
    }
    std::memcpy(o, no, sizeof(no));
    std::memcpy(u, nu, sizeof(nu));
}

hr_status read_camera(const std::string& path, hr_scene& sc) {
    std::ifstream in(path);
    if (!in) return io_error(HR_ERR_INVALID_ARG, "cannot read camera file %s", path.c_str());
    float rot[3] = {0, 0, 0};
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        std::stringstream ss(line);
        std::string key;
        if (!(ss >> key)) continue;
        if (key == "position") ss >> sc.pos[0] >> sc.pos[1] >> sc.pos[2];
        else if (key == "orientation") ss >> sc.orient[0] >> sc.orient[1] >> sc.orient[2];
        else if (key == "up") ss >> sc.up[0] >> sc.up[1] >> sc.up[2];
        else if (key == "rotation") ss >> rot[0] >> rot[1] >> rot[2];
        else if (key == "resX") ss >> sc.w;
        else if (key == "resY") ss >> sc.h;
        else if (key == "FOV") ss >> sc.fov;
    }
    camera_rotate(sc.orient, sc.up, rot);
    sc.has_camera = true;
    return HR_OK;
}

hr_status read_lights(const std::string& path, hr_scene& sc) {
    std::ifstream in(path);
    if (!in) return io_error(HR_ERR_INVALID_ARG, "cannot read light file %s", path.c_str());
    hr_scene::QuadLight cur;
    std::memset(&cur, 0, sizeof(cur));
    bool hp = false, hn = false, hi = false, h1 = false, h2 = false;
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        std::stringstream ss(line);
        std::string key;
        if (!(ss >> key)) continue;
        if (key == "position") { ss >> cur.position[0] >> cur.position[1] >> cur.position[2]; hp = true; }
        else if (key == "normal") { ss >> cur.normal[0] >> cur.normal[1] >> cur.normal[2]; hn = true; }
        else if (key == "intensity") { ss >> cur.intensity[0] >> cur.intensity[1] >> cur.intensity[2]; hi = true; }
        else if (key == "edge1") { ss >> cur.edge1[0] >> cur.edge1[1] >> cur.edge1[2]; h1 = true; }
        else if (key == "edge2") { ss >> cur.edge2[0] >> cur.edge2[1] >> cur.edge2[2]; h2 = true; }
        if (hp && hi && h1 && h2) {   // a complete light (LightSourceLoader.cpp:84-104)
            if (!hn) {
                const float* a = cur.edge1;
                const float* b = cur.edge2;
                float n[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
                const float len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                for (int k = 0; k < 3; ++k) cur.normal[k] = len > 0.0f ? n[k] / len : 0.0f;
            }
            sc.lights.push_back(cur);
            std::memset(&cur, 0, sizeof(cur));
            hp = hn = hi = h1 = h2 = false;
        }
    }
    return HR_OK;
}

// frame name of AnimationManager::read: the index zero-padded to the digit count of
// (frames - 1)
std::string frame_name(const std::string& prefix, const std::string& suffix, uint32_t frame, uint32_t frames) {
    int digits = 0;
    for (int n = (int)frames - 1; n > 0; n /= 10) ++digits;
    std::string id = std::to_string(frame);
    while ((int)id.size() < digits) id = "0" + id;
    return prefix + id + suffix;
}

// the normals and materials of one more OBJ file of a static scene, whose triangles follow
// tri_before earlier ones: normal indices move past the earlier normals, materials merge
// by name; triangles of files without them get sentinels (normals) or "Default"
hr_status append_extras(ObjExtras& acc, ObjExtras& ex, size_t tri_before, size_t tri_count) {
    if (!ex.normals.empty() || !acc.normals.empty()) {
        acc.nidx.resize(3 * tri_before, kNoNormal);
        if (ex.normals.empty()) {
            acc.nidx.resize(3 * (tri_before + tri_count), kNoNormal);
        } else {
            const size_t off = acc.normals.size() / 3;
            if (off + ex.normals.size() / 3 >= kNoNormal) return io_error(HR_ERR_INVALID_ARG, "too many normals");
            acc.normals.insert(acc.normals.end(), ex.normals.begin(), ex.normals.end());
            for (uint32_t x : ex.nidx) acc.nidx.push_back((uint32_t)(x + off));
        }
    }
    if (!ex.tri_mat.empty() || !acc.tri_mat.empty()) {
        if (acc.mat_names.empty()) {
            acc.mat_names.push_back("Default");
            acc.albedo.push_back(0.6774f);
        }
        acc.tri_mat.resize(tri_before, 0);
        if (ex.tri_mat.empty()) {
            acc.tri_mat.resize(tri_before + tri_count, 0);
        } else {
            std::vector<uint32_t> remap(ex.mat_names.size());
            for (size_t m = 0; m < ex.mat_names.size(); ++m) {
                const auto it = std::find(acc.mat_names.begin(), acc.mat_names.end(), ex.mat_names[m]);
                if (it != acc.mat_names.end()) {
                    remap[m] = (uint32_t)(it - acc.mat_names.begin());
                } else {
                    remap[m] = (uint32_t)acc.mat_names.size();
                    acc.mat_names.push_back(ex.mat_names[m]);
                    acc.albedo.push_back(ex.albedo[m]);
                }
            }
            for (uint32_t x : ex.tri_mat) acc.tri_mat.push_back(remap[x]);
        }
    }
    return HR_OK;
}

// the scene keeps the normals of `ns` (the first key frame's) and the materials of `ms`
hr_status take_extras(hr_scene& sc, ObjExtras& ns, ObjExtras& ms) {
    if (!ns.normals.empty()) {
        if (ns.nidx.size() != 3 * (size_t)sc.nt)
            return io_error(HR_ERR_INVALID_ARG, "the first key frame's normal indices do not match the triangles");
        if (!fill_geometric_normals(ns.normals, ns.nidx, sc.kf.data(), sc.idx))
            return io_error(HR_ERR_INVALID_ARG, "too many normals");
        sc.normals.swap(ns.normals);
        sc.nidx.swap(ns.nidx);
    }
    if (!ms.tri_mat.empty()) {
        if (ms.tri_mat.size() != sc.nt)
            return io_error(HR_ERR_INVALID_ARG, "the material list does not match the triangles");
        sc.albedo.swap(ms.albedo);
        sc.tri_mat.swap(ms.tri_mat);
    }
    return HR_OK;
}

hr_status finish_scene(hr_scene& sc, std::vector<std::vector<float>>& frames, std::vector<uint32_t>& idx) {
    if (frames.empty()) return io_error(HR_ERR_INVALID_ARG, "the scene has no geometry");
    const size_t nv3 = frames[0].size();
    for (const auto& f : frames)
        if (f.size() != nv3)
            return io_error(HR_ERR_INVALID_ARG, "key frames differ in vertex count (%zu vs %zu)", f.size() / 3, nv3 / 3);
    sc.nv = (uint32_t)(nv3 / 3);
    sc.nt = (uint32_t)(idx.size() / 3);
    sc.nkf = (uint32_t)frames.size();
    sc.kf.reserve(nv3 * frames.size());
    for (const auto& f : frames) sc.kf.insert(sc.kf.end(), f.begin(), f.end());
    sc.idx.swap(idx);
    return HR_OK;
}

// ---------------------------------------------------------------------------------
// PNG (RFC 2083) with stored deflate blocks (RFC 1950 / 1951)

uint32_t crc32_update(uint32_t crc, const uint8_t* p, size_t n) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? 0xEDB88320u ^ (c >> 1) : (c >> 1);
            table[i] = c;
        }
        init = true;
    }
    for (size_t i = 0; i < n; ++i) crc = table[(crc ^ p[i]) & 0xFFu] ^ (crc >> 8);
    return crc;
}

void put_be32(std::vector<uint8_t>& o, uint32_t x) {
    o.push_back((uint8_t)(x >> 24)); o.push_back((uint8_t)(x >> 16)); o.push_back((uint8_t)(x >> 8)); o.push_back((uint8_t)x);
}

void png_chunk(std::vector<uint8_t>& o, const char* type, const std::vector<uint8_t>& data) {
    put_be32(o, (uint32_t)data.size());
    const size_t at = o.size();
    o.insert(o.end(), type, type + 4);
    o.insert(o.end(), data.begin(), data.end());
    put_be32(o, crc32_update(0xFFFFFFFFu, o.data() + at, data.size() + 4) ^ 0xFFFFFFFFu);
}

hr_status write_png(const std::string& path, const float* rgb, int32_t w, int32_t h) {
    std::vector<uint8_t> raw;   // filter byte 0 + RGB per row
    raw.reserve((size_t)h * ((size_t)w * 3 + 1));
    for (int32_t y = 0; y < h; ++y) {
        raw.push_back(0);
        for (int32_t x = 0; x < w; ++x)
            for (int k = 0; k < 3; ++k) {
                float c = rgb[((size_t)y * w + x) * 3 + k];
                c = std::max(std::min(c, 1.0f), 0.0f);   // NaN -> 0
                raw.push_back((uint8_t)(c * 255.0f));
            }
    }
    std::vector<uint8_t> z = {0x78, 0x01};   // zlib header, no compression
    uint32_t a = 1, b = 0;                   // Adler-32
    for (size_t off = 0; off < raw.size() || off == 0;) {
        const size_t len = std::min<size_t>(65535, raw.size() - off);
        const bool last = off + len >= raw.size();
        z.push_back(last ? 1 : 0);
        z.push_back((uint8_t)len); z.push_back((uint8_t)(len >> 8));
        z.push_back((uint8_t)~len); z.push_back((uint8_t)(~len >> 8));
        z.insert(z.end(), raw.begin() + off, raw.begin() + off + len);
        for (size_t i = off; i < off + len; ++i) { a = (a + raw[i]) % 65521u; b = (b + a) % 65521u; }
        off += len;
        if (last) break;
    }
    put_be32(z, (b << 16) | a);
    std::vector<uint8_t> o = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1A, '\n'};
    std::vector<uint8_t> ihdr;
    put_be32(ihdr, (uint32_t)w);
    put_be32(ihdr, (uint32_t)h);
    ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});   // 8-bit RGB, deflate, no filter method, no interlace
    png_chunk(o, "IHDR", ihdr);
    png_chunk(o, "IDAT", z);
    png_chunk(o, "IEND", {});
    std::ofstream f(path, std::ios::binary);
    if (!f) return io_error(HR_ERR_INVALID_ARG, "cannot write %s", path.c_str());
    f.write((const char*)o.data(), (std::streamsize)o.size());
    return f ? HR_OK : io_error(HR_ERR_INVALID_ARG, "cannot write %s", path.c_str());
}

hr_status write_pfm(const std::string& path, const float* rgb, int32_t w, int32_t h) {
    std::ofstream f(path, std::ios::binary);
    if (!f) return io_error(HR_ERR_INVALID_ARG, "cannot write %s", path.c_str());
    f << "PF\n" << w << " " << h << "\n-1.0\n";   // little-endian floats, rows bottom to top
    for (int32_t y = h - 1; y >= 0; --y) f.write((const char*)(rgb + (size_t)y * w * 3), (std::streamsize)w * 12);
    return f ? HR_OK : io_error(HR_ERR_INVALID_ARG, "cannot write %s", path.c_str());
}

}  // namespace

extern "C" {

const char* hr_io_last_error(void) { return g_err.c_str(); }

hr_status hr_scene_load_obj(const char* path, int32_t threads, hr_scene** out) {
    if (!path || !out) return io_error(HR_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    hr_scene* sc = new (std::nothrow) hr_scene();
    if (!sc) return HR_ERR_OUT_OF_MEMORY;
    std::vector<std::vector<float>> frames(1);
    std::vector<uint32_t> idx;
    ObjExtras ex;
    hr_status st = read_obj(path, threads, frames[0], idx, &ex);
    if (st == HR_OK) st = finish_scene(*sc, frames, idx);
    if (st == HR_OK) st = take_extras(*sc, ex, ex);
    if (st != HR_OK) { delete sc; return st; }
    *out = sc;
    return HR_OK;
}

hr_status hr_scene_load(const char* cfg, int32_t threads, hr_scene** out) {
    if (!cfg || !out) return io_error(HR_ERR_INVALID_ARG, "null argument");
    *out = nullptr;
    std::ifstream in(cfg);
    if (!in) return io_error(HR_ERR_INVALID_ARG, "cannot read %s", cfg);
    const std::string base = dir_of(cfg);
    std::vector<std::string> objs;
    std::string prefix, suffix, camera, light;
    uint32_t nframes = 0;
    float step = 0.0f;
    std::string line;
    while (std::getline(in, line)) {
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        const size_t eq = line.find('=');
        if (eq == std::string::npos) continue;
        const std::string key = trim(line.substr(0, eq));
        const std::string val = trim(line.substr(eq + 1));
        if (key == "obj" || key == "scene") objs.push_back(val);
        else if (key == "camera" || key == "view" || key == "cam") camera = val;
        else if (key == "frame prefix" || key == "frameprefix" || key == "framename") prefix = val;
        else if (key == "frame suffix" || key == "framesuffix") suffix = val;
        else if (key == "frame number" || key == "number" || key == "framenumber" || key == "number of frames")
            nframes = (uint32_t)std::strtoul(val.c_str(), nullptr, 10);
        else if (key == "frame step" || key == "framestep" || key == "step size")
            step = std::strtof(val.c_str(), nullptr);
        else if (key == "light sources" || key == "light source" || key == "light" || key == "lights")
            light = val;
        // camera path, instances and unknown keys: not used by the hot path
    }
    hr_scene* sc = new (std::nothrow) hr_scene();
    if (!sc) return HR_ERR_OUT_OF_MEMORY;
    std::vector<std::vector<float>> frames;
    std::vector<uint32_t> idx;
    ObjExtras first, last;
    hr_status st = HR_OK;
    if (nframes > 0 && (!prefix.empty() || !suffix.empty())) {
        // key frames (AnimationManager::read): the last frame's triangles and materials are
        // kept, the first frame's normals (RTEngine::upload takes the normals of its first
        // frame, RTEngine.cu:205-209; WFObjectUploader.h:121-250)
        for (uint32_t k = 0; k < nframes && st == HR_OK; ++k) {
            std::vector<float> v;
            st = read_obj(resolve(frame_name(prefix, suffix, k, nframes), base), threads, v, idx,
                          k == 0 ? &first : &last);
            frames.push_back(std::move(v));
        }
    } else {
        // one static frame: the listed OBJ files concatenated
        frames.emplace_back();
        for (size_t i = 0; i < objs.size() && st == HR_OK; ++i) {
            std::vector<float> v;
            std::vector<uint32_t> fi;
            ObjExtras ex;
            st = read_obj(resolve(objs[i], base), threads, v, fi, &ex);
            if (st == HR_OK) st = append_extras(first, ex, (uint32_t)(idx.size() / 3), (uint32_t)(fi.size() / 3));
            const uint32_t off = (uint32_t)(frames[0].size() / 3);
            for (uint32_t& x : fi) x += off;
            frames[0].insert(frames[0].end(), v.begin(), v.end());
            idx.insert(idx.end(), fi.begin(), fi.end());
        }
        nframes = 1;
    }
    sc->frame_step = step;
    if (st == HR_OK) st = finish_scene(*sc, frames, idx);
    if (st == HR_OK) st = take_extras(*sc, first, nframes > 1 ? last : first);
    if (st == HR_OK && !camera.empty()) st = read_camera(resolve(camera, base), *sc);
    if (st == HR_OK && !light.empty() && file_exists(resolve(light, base))) st = read_lights(resolve(light, base), *sc);
    if (st != HR_OK) { delete sc; return st; }
    *out = sc;
    return HR_OK;
}

void hr_scene_free(hr_scene* sc) { delete sc; }

hr_status hr_scene_get_info(const hr_scene* sc, hr_scene_info* info) {
    if (!sc || !info) return io_error(HR_ERR_INVALID_ARG, "null argument");
    info->num_vertices = sc->nv;
    info->num_triangles = sc->nt;
    info->num_keyframes = sc->nkf;
    info->frame_step = sc->frame_step;
    info->has_camera = sc->has_camera ? 1 : 0;
    for (int k = 0; k < 3; ++k) {
        info->cam_position[k] = sc->pos[k]; info->cam_orientation[k] = sc->orient[k]; info->cam_up[k] = sc->up[k];
    }
    info->cam_fov_deg = sc->fov;
    info->width = sc->w;
    info->height = sc->h;
    info->num_lights = (uint32_t)sc->lights.size();
    info->num_normals = (uint32_t)(sc->normals.size() / 3);
    info->num_materials = (uint32_t)sc->albedo.size();
    return HR_OK;
}

const float* hr_scene_keyframes(const hr_scene* sc) { return sc ? sc->kf.data() : nullptr; }
const uint32_t* hr_scene_indices(const hr_scene* sc) { return sc ? sc->idx.data() : nullptr; }
const float* hr_scene_normals(const hr_scene* sc) { return sc && !sc->normals.empty() ? sc->normals.data() : nullptr; }
const uint32_t* hr_scene_normal_indices(const hr_scene* sc) {
    return sc && !sc->normals.empty() ? sc->nidx.data() : nullptr;
}
const float* hr_scene_material_albedo(const hr_scene* sc) {
    return sc && !sc->albedo.empty() ? sc->albedo.data() : nullptr;
}
const uint32_t* hr_scene_triangle_materials(const hr_scene* sc) {
    return sc && !sc->albedo.empty() ? sc->tri_mat.data() : nullptr;
}

hr_status hr_scene_get_light(const hr_scene* sc, uint32_t i, float pos[3], float e1[3], float e2[3], float n[3],
                             float inten[3]) {
    if (!sc || i >= sc->lights.size()) return io_error(HR_ERR_INVALID_ARG, "no light %u", i);
    const hr_scene::QuadLight& L = sc->lights[i];
    for (int k = 0; k < 3; ++k) {
        if (pos) pos[k] = L.position[k];
        if (e1) e1[k] = L.edge1[k];
        if (e2) e2[k] = L.edge2[k];
        if (n) n[k] = L.normal[k];
        if (inten) inten[k] = L.intensity[k];
    }
    return HR_OK;
}

hr_status hr_scene_upload(hr_ctx* ctx, const hr_scene* sc) {
    if (!ctx || !sc) return io_error(HR_ERR_INVALID_ARG, "null argument");
    hr_status st = hr_set_keyframes(ctx, sc->kf.data(), sc->nkf, sc->nv, sc->idx.data(), sc->nt);
    if (st != HR_OK) return st;
    if (sc->has_camera && sc->w > 0 && sc->h > 0 &&
        (st = hr_set_camera(ctx, sc->pos, sc->orient, sc->up, sc->fov, sc->w, sc->h)) != HR_OK)
        return st;
    if (!sc->lights.empty()) {   // every light, emission = mean intensity (scalar radiance)
        const size_t n = std::min(sc->lights.size(), (size_t)64);
        std::vector<float> pos(3 * n), e1(3 * n), e2(3 * n), nrm(3 * n), em(n);
        for (size_t k = 0; k < n; ++k) {
            const hr_scene::QuadLight& L = sc->lights[k];
            for (int i = 0; i < 3; ++i) {
                pos[3 * k + i] = L.position[i]; e1[3 * k + i] = L.edge1[i]; e2[3 * k + i] = L.edge2[i];
                nrm[3 * k + i] = L.normal[i];
            }
            em[k] = (L.intensity[0] + L.intensity[1] + L.intensity[2]) / 3.0f;
        }
        if ((st = hr_set_lights(ctx, (uint32_t)n, pos.data(), e1.data(), e2.data(), nrm.data(), em.data())) != HR_OK)
            return st;
    }
    // the mesh's shading normals and materials, or none (a scene without them must not
    // keep an earlier scene's)
    st = sc->normals.empty() ? hr_set_normals(ctx, nullptr, 0, nullptr)
                             : hr_set_normals(ctx, sc->normals.data(), (uint32_t)(sc->normals.size() / 3), sc->nidx.data());
    if (st != HR_OK) return st;
    st = sc->albedo.empty() ? hr_set_materials(ctx, nullptr, 0, nullptr)
                            : hr_set_materials(ctx, sc->albedo.data(), (uint32_t)sc->albedo.size(), sc->tri_mat.data());
    if (st != HR_OK) return st;
    return hr_set_frame_time(ctx, 0.0f, 0.0f);
}

hr_status hr_rays_file_count(const char* path, uint32_t* n) {
    if (!path || !n) return io_error(HR_ERR_INVALID_ARG, "null argument");
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) return io_error(HR_ERR_INVALID_ARG, "cannot read %s", path);
    const std::streamoff sz = f.tellg();
    if (sz < 0 || sz % 24 != 0) return io_error(HR_ERR_INVALID_ARG, "%s: size is not a multiple of 24 bytes", path);
    if (sz / 24 > 0xffffffffll) return io_error(HR_ERR_INVALID_ARG, "%s: too many rays", path);
    *n = (uint32_t)(sz / 24);
    return HR_OK;
}

hr_status hr_rays_file_read(const char* path, float* org_dir, uint32_t n) {
    uint32_t have = 0;
    hr_status st = hr_rays_file_count(path, &have);
    if (st != HR_OK) return st;
    if (!org_dir || n != have) return io_error(HR_ERR_INVALID_ARG, "%s holds %u rays, %u asked", path, have, n);
    std::ifstream f(path, std::ios::binary);
    f.read((char*)org_dir, (std::streamsize)n * 24);
    return f ? HR_OK : io_error(HR_ERR_INVALID_ARG, "cannot read %s", path);
}

hr_status hr_rays_file_write(const char* path, const float* org, const float* dir, uint32_t n) {
    if (!path || (n && (!org || !dir))) return io_error(HR_ERR_INVALID_ARG, "null argument");
    std::ofstream f(path, std::ios::binary);
    if (!f) return io_error(HR_ERR_INVALID_ARG, "cannot write %s", path);
    std::vector<float> buf((size_t)std::min<uint32_t>(n, 1u << 20) * 6);
    for (uint32_t b = 0; b < n; b += 1u << 20) {
        const uint32_t m = std::min<uint32_t>(n - b, 1u << 20);
        for (uint32_t i = 0; i < m; ++i)
            for (int k = 0; k < 3; ++k) {
                buf[6 * (size_t)i + k] = org[3 * ((size_t)b + i) + k];
                buf[6 * (size_t)i + 3 + k] = dir[3 * ((size_t)b + i) + k];
            }
        f.write((const char*)buf.data(), (std::streamsize)m * 24);
    }
    return f ? HR_OK : io_error(HR_ERR_INVALID_ARG, "cannot write %s", path);
}

hr_status hr_hits_file_write(const char* path, const int32_t* id, const float* t, const float* u, const float* v,
                             uint32_t n) {
    if (!path || (n && (!id || !t || !u || !v))) return io_error(HR_ERR_INVALID_ARG, "null argument");
    std::ofstream f(path, std::ios::binary);
    if (!f) return io_error(HR_ERR_INVALID_ARG, "cannot write %s", path);
    for (uint32_t i = 0; i < n; ++i) {
        f.write((const char*)(id + i), 4);
        f.write((const char*)(t + i), 4);
        f.write((const char*)(u + i), 4);
        f.write((const char*)(v + i), 4);
    }
    return f ? HR_OK : io_error(HR_ERR_INVALID_ARG, "cannot write %s", path);
}

// The reference's instances file (WFObject::loadInstances, WFObjectReader.cpp:762-825):
// "obj_id" starts an instance (identity map, empty box), "m_row_0..2" give the rows of
// the world -> object map (rotation column entries, then translation), "AABB_min" /
// "AABB_max" the world box; '#' starts a comment.
hr_status hr_instances_file_read(const char* path, hr_instance* inst, uint32_t cap, uint32_t* n_out) {
    if (!path || !n_out) return io_error(HR_ERR_INVALID_ARG, "null argument");
    std::ifstream in(path);
    if (!in) return io_error(HR_ERR_INVALID_ARG, "cannot read instances file %s", path);
    std::string line;
    size_t lineno = 0;
    uint32_t n = 0;
    hr_instance cur{};
    auto flush = [&]() {
        if (n > 0 && inst && n - 1 < cap) inst[n - 1] = cur;
    };
    while (std::getline(in, line)) {
        ++lineno;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line = line.substr(0, hash);
        std::stringstream ss(line);
        std::string key;
        if (!(ss >> key)) continue;
        if (key == "obj_id") {
            flush();
            cur = hr_instance{};
            cur.m[0] = cur.m[5] = cur.m[10] = 1.0f;
            for (int k = 0; k < 3; ++k) { cur.bmin[k] = FLT_MAX; cur.bmax[k] = -FLT_MAX; }
            long long id = -1;
            if (!(ss >> id) || id < 0 || id > 0xffffffffLL)
                return io_error(HR_ERR_INVALID_ARG, "%s line %zu: bad obj_id", path, lineno);
            cur.object = (uint32_t)id;
            ++n;
            continue;
        }
        float* dst = nullptr;
        int cnt = 0;
        if (key == "m_row_0") { dst = cur.m; cnt = 4; }
        else if (key == "m_row_1") { dst = cur.m + 4; cnt = 4; }
        else if (key == "m_row_2") { dst = cur.m + 8; cnt = 4; }
        else if (key == "AABB_min") { dst = cur.bmin; cnt = 3; }
        else if (key == "AABB_max") { dst = cur.bmax; cnt = 3; }
        else continue;   // other keys are ignored, as the reference does
        if (n == 0) return io_error(HR_ERR_INVALID_ARG, "%s line %zu: %s before obj_id", path, lineno, key.c_str());
        for (int k = 0; k < cnt; ++k)
            if (!(ss >> dst[k])) return io_error(HR_ERR_INVALID_ARG, "%s line %zu: %s needs %d numbers", path, lineno,
                                                 key.c_str(), cnt);
    }
    flush();
    *n_out = n;
    return HR_OK;
}

// ObjWriter::writeInstance (WFObjWriter.cpp:94-111) layout; numbers with 9 significant
// digits so that a file read back gives the same floats
hr_status hr_instances_file_write(const char* path, const hr_instance* inst, uint32_t n) {
    if (!path || (n && !inst)) return io_error(HR_ERR_INVALID_ARG, "null argument");
    FILE* f = std::fopen(path, "w");
    if (!f) return io_error(HR_ERR_INVALID_ARG, "cannot write %s", path);
    for (uint32_t i = 0; i < n; ++i) {
        const hr_instance& r = inst[i];
        std::fprintf(f, "#new instance#\nobj_id %u\n", r.object);
        for (int row = 0; row < 3; ++row)
            std::fprintf(f, "m_row_%d %.9g %.9g %.9g %.9g\n", row, r.m[4 * row], r.m[4 * row + 1], r.m[4 * row + 2],
                         r.m[4 * row + 3]);
        std::fprintf(f, "AABB_min %.9g %.9g %.9g\nAABB_max %.9g %.9g %.9g\n", r.bmin[0], r.bmin[1], r.bmin[2], r.bmax[0],
                     r.bmax[1], r.bmax[2]);
    }
    const bool ok = std::ferror(f) == 0;
    std::fclose(f);
    return ok ? HR_OK : io_error(HR_ERR_INVALID_ARG, "cannot write %s", path);
}

hr_status hr_image_write(const char* path, const float* rgb, int32_t w, int32_t h, int32_t format) {
    if (!path || !rgb || w <= 0 || h <= 0) return io_error(HR_ERR_INVALID_ARG, "bad image arguments");
    if (format == HR_IMAGE_PNG) return write_png(path, rgb, w, h);
    if (format == HR_IMAGE_PFM) return write_pfm(path, rgb, w, h);
    return io_error(HR_ERR_INVALID_ARG, "unknown image format %d", format);
}

}  // extern "C"
