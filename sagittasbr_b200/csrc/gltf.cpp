// gltf.cpp -- glTF 2.0 mesh input (.gltf with external or data: buffers, and
// binary .glb), the model formats the reference reads through tinygltf
// (src/modelLoader.cpp:286-413), plus the extension dispatch of loadModel
// (src/modelLoader.cpp:421-450).
//
// What is read follows the reference loader: every primitive of every mesh in
// file order (node transforms are not applied), primitives whose mode is
// TRIANGLES (the default when absent), POSITION accessors of FLOAT components
// (others skip the primitive), indices of unsigned byte / short / int components
// (a primitive without indices uses its vertices in order), each primitive's
// indices offset by the vertices read before it.  Byte strides, accessor and
// buffer-view offsets are honoured; sparse accessors are not supported (the
// primitive is rejected with SBR_ERR_PARSE).
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "common.hpp"

using namespace sbr;

namespace {

// ------------------------------------------------------------------ JSON
struct JVal {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;

    const JVal* get(const char* key) const {
        if (kind != OBJ) return nullptr;
        for (const auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    double num_or(const char* key, double dflt) const {
        const JVal* v = get(key);
        return v && v->kind == NUM ? v->num : dflt;
    }
};

struct JParser {
    const char* p;
    const char* end;
    std::string err;

    void ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
    }
    bool lit(const char* s) {
        size_t n = std::strlen(s);
        if ((size_t)(end - p) < n || std::strncmp(p, s, n) != 0) return false;
        p += n;
        return true;
    }
    static void utf8(std::string& o, unsigned cp) {
        if (cp < 0x80) o += char(cp);
        else if (cp < 0x800) { o += char(0xC0 | (cp >> 6)); o += char(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000) { o += char(0xE0 | (cp >> 12)); o += char(0x80 | ((cp >> 6) & 0x3F)); o += char(0x80 | (cp & 0x3F)); }
        else { o += char(0xF0 | (cp >> 18)); o += char(0x80 | ((cp >> 12) & 0x3F)); o += char(0x80 | ((cp >> 6) & 0x3F)); o += char(0x80 | (cp & 0x3F)); }
    }
    bool string(std::string& out) {
        if (p >= end || *p != '"') return false;
        ++p;
        while (p < end && *p != '"') {
            if (*p == '\\') {
                if (++p >= end) return false;
                switch (*p) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        if (end - p < 5) return false;
                        unsigned cp = (unsigned)std::strtoul(std::string(p + 1, p + 5).c_str(), nullptr, 16);
                        p += 4;
                        utf8(out, cp);
                        break;
                    }
                    default: return false;
                }
                ++p;
            } else {
                out += *p++;
            }
        }
        if (p >= end) return false;
        ++p;
        return true;
    }
    bool value(JVal& v, int depth) {
        if (depth > 256) return false;
        ws();
        if (p >= end) return false;
        const char c = *p;
        if (c == '{') {
            v.kind = JVal::OBJ;
            ++p;
            ws();
            if (p < end && *p == '}') { ++p; return true; }
            for (;;) {
                ws();
                std::string k;
                if (!string(k)) return false;
                ws();
                if (p >= end || *p != ':') return false;
                ++p;
                v.obj.emplace_back(std::move(k), JVal{});
                if (!value(v.obj.back().second, depth + 1)) return false;
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == '}') { ++p; return true; }
                return false;
            }
        }
        if (c == '[') {
            v.kind = JVal::ARR;
            ++p;
            ws();
            if (p < end && *p == ']') { ++p; return true; }
            for (;;) {
                v.arr.emplace_back();
                if (!value(v.arr.back(), depth + 1)) return false;
                ws();
                if (p < end && *p == ',') { ++p; continue; }
                if (p < end && *p == ']') { ++p; return true; }
                return false;
            }
        }
        if (c == '"') { v.kind = JVal::STR; return string(v.str); }
        if (lit("true")) { v.kind = JVal::BOOL; v.b = true; return true; }
        if (lit("false")) { v.kind = JVal::BOOL; v.b = false; return true; }
        if (lit("null")) { v.kind = JVal::NUL; return true; }
        char* e = nullptr;
        std::string tmp(p, (size_t)std::min<ptrdiff_t>(end - p, 64));
        v.num = std::strtod(tmp.c_str(), &e);
        if (e == tmp.c_str()) return false;
        v.kind = JVal::NUM;
        p += (e - tmp.c_str());
        return true;
    }
};

bool parse_json(const char* b, size_t n, JVal& out) {
    JParser ps{b, b + n, {}};
    if (!ps.value(out, 0)) return false;
    ps.ws();
    return ps.p == ps.end;
}

// ------------------------------------------------------------- buffers
bool base64(const std::string& s, size_t from, std::vector<unsigned char>& out) {
    auto val = [](char c) -> int {
        if (c >= 'A' && c <= 'Z') return c - 'A';
        if (c >= 'a' && c <= 'z') return c - 'a' + 26;
        if (c >= '0' && c <= '9') return c - '0' + 52;
        if (c == '+') return 62;
        if (c == '/') return 63;
        return -1;
    };
    unsigned acc = 0;
    int bits = 0;
    for (size_t i = from; i < s.size(); ++i) {
        const char c = s[i];
        if (c == '=') break;
        const int d = val(c);
        if (d < 0) {
            if (std::isspace((unsigned char)c)) continue;
            return false;
        }
        acc = (acc << 6) | (unsigned)d;
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out.push_back((unsigned char)((acc >> bits) & 0xFF));
        }
    }
    return true;
}

bool read_file(const std::string& path, std::vector<unsigned char>& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f.is_open()) return false;
    out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

std::string dir_of(const std::string& path) {
    const size_t s = path.find_last_of("/\\");
    return s == std::string::npos ? std::string() : path.substr(0, s + 1);
}

bool has_ext(std::string s, const char* ext) {
    for (auto& ch : s) ch = (char)std::tolower((unsigned char)ch);
    const size_t n = std::strlen(ext);
    return s.size() >= n && s.compare(s.size() - n, n, ext) == 0;
}

struct Gltf {
    JVal doc;
    std::vector<std::vector<unsigned char>> buffers;
};

sbr_status load_doc(const std::string& path, Gltf& g) {
    std::vector<unsigned char> raw;
    if (!read_file(path, raw)) return fail(SBR_ERR_IO, "cannot open " + path);
    std::vector<unsigned char> bin;
    bool glb = false;
    const unsigned char* json = raw.data();
    size_t json_len = raw.size();
    if (raw.size() >= 12 && std::memcmp(raw.data(), "glTF", 4) == 0) {
        glb = true;
        uint32_t version, length;
        std::memcpy(&version, raw.data() + 4, 4);
        std::memcpy(&length, raw.data() + 8, 4);
        if (version != 2 || length > raw.size()) return fail(SBR_ERR_PARSE, "bad GLB header in " + path);
        size_t off = 12;
        json = nullptr;
        while (off + 8 <= length) {
            uint32_t clen, ctype;
            std::memcpy(&clen, raw.data() + off, 4);
            std::memcpy(&ctype, raw.data() + off + 4, 4);
            if (off + 8 + (size_t)clen > length) return fail(SBR_ERR_PARSE, "truncated GLB chunk in " + path);
            if (ctype == 0x4E4F534Au && !json) { json = raw.data() + off + 8; json_len = clen; }
            else if (ctype == 0x004E4942u && bin.empty()) bin.assign(raw.data() + off + 8, raw.data() + off + 8 + clen);
            off += 8 + (size_t)((clen + 3) & ~3u);
        }
        if (!json) return fail(SBR_ERR_PARSE, "GLB without a JSON chunk: " + path);
    }
    if (!parse_json((const char*)json, json_len, g.doc) || g.doc.kind != JVal::OBJ)
        return fail(SBR_ERR_PARSE, "malformed glTF JSON in " + path);
    const JVal* bufs = g.doc.get("buffers");
    if (bufs && bufs->kind == JVal::ARR) {
        for (size_t k = 0; k < bufs->arr.size(); ++k) {
            const JVal& b = bufs->arr[k];
            const JVal* uri = b.get("uri");
            std::vector<unsigned char> data;
            if (!uri) {
                if (!(glb && k == 0)) return fail(SBR_ERR_PARSE, "buffer without uri in " + path);
                data = bin;
            } else if (uri->kind == JVal::STR && uri->str.compare(0, 5, "data:") == 0) {
                const size_t comma = uri->str.find(',');
                if (comma == std::string::npos || uri->str.find(";base64") == std::string::npos ||
                    !base64(uri->str, comma + 1, data))
                    return fail(SBR_ERR_PARSE, "unsupported data URI in " + path);
            } else if (uri->kind == JVal::STR) {
                if (!read_file(dir_of(path) + uri->str, data))
                    return fail(SBR_ERR_IO, "cannot open buffer " + uri->str + " of " + path);
            } else {
                return fail(SBR_ERR_PARSE, "bad buffer uri in " + path);
            }
            const double want = b.num_or("byteLength", -1.0);
            if (want < 0 || (double)data.size() < want) return fail(SBR_ERR_PARSE, "buffer shorter than byteLength");
            g.buffers.push_back(std::move(data));
        }
    }
    return SBR_OK;
}

// Locates an accessor's elements: base pointer, element stride and count, with
// every byte of every element checked against its buffer.
sbr_status accessor_span(const Gltf& g, int index, int comps, int comp_size, const unsigned char** base,
                         size_t* stride, size_t* count, int* comp_type) {
    const JVal* accs = g.doc.get("accessors");
    const JVal* views = g.doc.get("bufferViews");
    if (!accs || accs->kind != JVal::ARR || index < 0 || (size_t)index >= accs->arr.size())
        return fail(SBR_ERR_PARSE, "accessor index out of range");
    const JVal& a = accs->arr[index];
    if (a.get("sparse")) return fail(SBR_ERR_PARSE, "sparse accessors are not supported");
    *comp_type = (int)a.num_or("componentType", -1);
    *count = (size_t)a.num_or("count", 0);
    const int bv = (int)a.num_or("bufferView", -1);
    if (!views || views->kind != JVal::ARR || bv < 0 || (size_t)bv >= views->arr.size())
        return fail(SBR_ERR_PARSE, "accessor without a valid bufferView");
    const JVal& v = views->arr[bv];
    const int bi = (int)v.num_or("buffer", -1);
    if (bi < 0 || (size_t)bi >= g.buffers.size()) return fail(SBR_ERR_PARSE, "bufferView buffer out of range");
    const size_t voff = (size_t)v.num_or("byteOffset", 0), vlen = (size_t)v.num_or("byteLength", 0);
    const size_t aoff = (size_t)a.num_or("byteOffset", 0);
    size_t st = (size_t)v.num_or("byteStride", 0);
    if (st == 0) st = (size_t)comps * (size_t)comp_size;
    const std::vector<unsigned char>& buf = g.buffers[bi];
    if (voff + vlen > buf.size()) return fail(SBR_ERR_PARSE, "bufferView exceeds its buffer");
    if (*count > 0 && aoff + (*count - 1) * st + (size_t)comps * comp_size > vlen)
        return fail(SBR_ERR_PARSE, "accessor exceeds its bufferView");
    *base = buf.data() + voff + aoff;
    *stride = st;
    return SBR_OK;
}

int type_components(const JVal& acc) {
    const JVal* t = acc.get("type");
    if (!t || t->kind != JVal::STR) return 0;
    static const std::map<std::string, int> n{{"SCALAR", 1}, {"VEC2", 2}, {"VEC3", 3}, {"VEC4", 4},
                                              {"MAT2", 4}, {"MAT3", 9}, {"MAT4", 16}};
    auto it = n.find(t->str);
    return it == n.end() ? 0 : it->second;
}

sbr_status emit(std::vector<float>& V, std::vector<uint32_t>& T, float** xyz, size_t* nverts, uint32_t** tri_idx,
                size_t* ntris, const std::string& path) {
    if (T.size() < 3) return fail(SBR_ERR_EMPTY_MESH, "no triangles in " + path);
    T.resize(T.size() - T.size() % 3);
    *xyz = (float*)std::malloc(std::max<size_t>(1, V.size()) * sizeof(float));
    *tri_idx = (uint32_t*)std::malloc(T.size() * sizeof(uint32_t));
    if (!*xyz || !*tri_idx) {
        std::free(*xyz);
        std::free(*tri_idx);
        *xyz = nullptr;
        *tri_idx = nullptr;
        return fail(SBR_ERR_OOM, "host allocation failed");
    }
    if (!V.empty()) std::memcpy(*xyz, V.data(), V.size() * sizeof(float));
    std::memcpy(*tri_idx, T.data(), T.size() * sizeof(uint32_t));
    *nverts = V.size() / 3;
    *ntris = T.size() / 3;
    return SBR_OK;
}

}  // namespace

extern "C" {

sbr_status sbr_load_gltf(const char* path, float** xyz, size_t* nverts, uint32_t** tri_idx, size_t* ntris) {
    if (!path || !xyz || !nverts || !tri_idx || !ntris) return fail(SBR_ERR_INVALID_ARG, "null argument");
    *xyz = nullptr;
    *tri_idx = nullptr;
    *nverts = *ntris = 0;
    Gltf g;
    sbr_status st = load_doc(path, g);
    if (st != SBR_OK) return st;
    std::vector<float> V;
    std::vector<uint32_t> T;
    const JVal* meshes = g.doc.get("meshes");
    const JVal* accs = g.doc.get("accessors");
    if (meshes && meshes->kind == JVal::ARR) {
        for (const JVal& m : meshes->arr) {
            const JVal* prims = m.get("primitives");
            if (!prims || prims->kind != JVal::ARR) continue;
            for (const JVal& pr : prims->arr) {
                if ((int)pr.num_or("mode", 4) != 4) continue;  // TRIANGLES only
                const JVal* attrs = pr.get("attributes");
                const JVal* pos = attrs ? attrs->get("POSITION") : nullptr;
                if (!pos || pos->kind != JVal::NUM || !accs || accs->kind != JVal::ARR) continue;
                const int pa = (int)pos->num;
                if (pa < 0 || (size_t)pa >= accs->arr.size()) return fail(SBR_ERR_PARSE, "POSITION accessor out of range");
                const int pcomps = type_components(accs->arr[pa]);
                if ((int)accs->arr[pa].num_or("componentType", -1) != 5126 || pcomps <= 0) continue;  // FLOAT
                const unsigned char* base;
                size_t stride, count;
                int ctype;
                st = accessor_span(g, pa, pcomps, 4, &base, &stride, &count, &ctype);
                if (st != SBR_OK) return st;
                if (count == 0) continue;
                const uint32_t first = (uint32_t)(V.size() / 3);
                for (size_t i = 0; i < count; ++i) {
                    float c[3] = {0.0f, 0.0f, 0.0f};
                    std::memcpy(c, base + i * stride, sizeof(float) * (size_t)std::min(3, pcomps));
                    V.insert(V.end(), c, c + 3);
                }
                const JVal* ind = pr.get("indices");
                if (ind && ind->kind == JVal::NUM) {
                    const int ia = (int)ind->num;
                    if (ia < 0 || (size_t)ia >= accs->arr.size()) return fail(SBR_ERR_PARSE, "indices accessor out of range");
                    const int it = (int)accs->arr[ia].num_or("componentType", -1);
                    const int isz = it == 5121 ? 1 : it == 5123 ? 2 : it == 5125 ? 4 : 0;
                    if (isz == 0) return fail(SBR_ERR_PARSE, "unsupported index component type");
                    st = accessor_span(g, ia, 1, isz, &base, &stride, &count, &ctype);
                    if (st != SBR_OK) return st;
                    for (size_t i = 0; i < count; ++i) {
                        uint32_t k = 0;
                        if (isz == 1) k = base[i * stride];
                        else if (isz == 2) { uint16_t s; std::memcpy(&s, base + i * stride, 2); k = s; }
                        else std::memcpy(&k, base + i * stride, 4);
                        if ((size_t)k >= V.size() / 3 - first) return fail(SBR_ERR_BAD_INDEX, "glTF index out of range");
                        T.push_back(first + k);
                    }
                } else {
                    for (size_t i = 0; i < count; ++i) T.push_back(first + (uint32_t)i);
                }
            }
        }
    }
    return emit(V, T, xyz, nverts, tri_idx, ntris, path);
}

sbr_status sbr_load_model(const char* path, float** xyz, size_t* nverts, uint32_t** tri_idx, size_t* ntris) {
    if (!path) return fail(SBR_ERR_INVALID_ARG, "null path");
    if (has_ext(path, ".obj")) return sbr_load_obj(path, xyz, nverts, tri_idx, ntris);
    if (has_ext(path, ".gltf") || has_ext(path, ".glb")) return sbr_load_gltf(path, xyz, nverts, tri_idx, ntris);
    return fail(SBR_ERR_UNSUPPORTED, std::string("Unsupported file extension for \"") + path + "\"");
}

}  // extern "C"
