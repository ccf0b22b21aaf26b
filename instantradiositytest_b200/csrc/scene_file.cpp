// scene_file.cpp — the scene-format loader: Scene::load and Scene::validate
// (src/scene.rs:157-382) for a version-1 manifest (JSON) and its binary
// files, into a workload whose meshes are triangle lists with their SDF
// fields, ready for the G-buffer producer, the VPL generator and the hot path.
//
// The manifest is read as serde reads it into the reference's structs
// (src/scene.rs:11-135): fields in any order, unknown fields ignored except
// in `transform`, defaults for `base_color_srgb` (true), `normal_strength`
// (1), `texture_channels` ([0; 4]), light `direction` (0) and
// `angle_radians` (0); Vec3 and Quat are JSON arrays (x, y, z[, w]).  The
// checks and their order follow Scene::validate and the per-mesh loads; the
// error text names the same condition.  Textured materials pass validation
// (the texture files must exist) but are rejected afterwards: the input
// producers here shade with the material constants only.
#include <sys/stat.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <new>
#include <set>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

#include "workload.h"

namespace {

// ------------------------------------------------------------------ JSON
struct JVal {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0;
    bool integer = false;  // the literal had no fraction or exponent
    bool negative = false;
    uint64_t u = 0;        // magnitude of an integer literal (saturated flag below)
    bool u_overflow = false;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;

    const JVal* get(const char* key) const {
        for (const auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
};

struct Fail {
    std::string msg;
};

class Parser {
public:
    Parser(const char* s, size_t n) : p_(s), b_(s), e_(s + n) {}
    JVal document() {
        JVal v = value(0);
        ws();
        if (p_ != e_) fail("trailing characters");
        return v;
    }

private:
    const char *p_, *b_, *e_;

    [[noreturn]] void fail(const char* what) {
        size_t line = 1, col = 1;
        for (const char* q = b_; q < p_ && q < e_; q++) {
            if (*q == '\n') {
                line++;
                col = 1;
            } else {
                col++;
            }
        }
        std::ostringstream os;
        os << what << " at line " << line << " column " << col;
        throw Fail{os.str()};
    }
    void ws() {
        while (p_ < e_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) p_++;
    }
    bool lit(const char* w) {
        size_t n = std::strlen(w);
        if ((size_t)(e_ - p_) >= n && std::memcmp(p_, w, n) == 0) {
            p_ += n;
            return true;
        }
        return false;
    }
    JVal value(int depth) {
        if (depth > 128) fail("recursion limit exceeded");
        ws();
        if (p_ == e_) fail("EOF while parsing a value");
        JVal v;
        char c = *p_;
        if (c == '{') {
            v.kind = JVal::Obj;
            p_++;
            ws();
            if (p_ < e_ && *p_ == '}') {
                p_++;
                return v;
            }
            for (;;) {
                ws();
                if (p_ == e_ || *p_ != '"') fail("key must be a string");
                std::string k = string();
                ws();
                if (p_ == e_ || *p_ != ':') fail("expected `:`");
                p_++;
                for (const auto& kv : v.obj)
                    if (kv.first == k) fail(("duplicate field `" + k + "`").c_str());
                v.obj.emplace_back(std::move(k), value(depth + 1));
                ws();
                if (p_ < e_ && *p_ == ',') {
                    p_++;
                    continue;
                }
                if (p_ < e_ && *p_ == '}') {
                    p_++;
                    return v;
                }
                fail("expected `,` or `}`");
            }
        }
        if (c == '[') {
            v.kind = JVal::Arr;
            p_++;
            ws();
            if (p_ < e_ && *p_ == ']') {
                p_++;
                return v;
            }
            for (;;) {
                v.arr.push_back(value(depth + 1));
                ws();
                if (p_ < e_ && *p_ == ',') {
                    p_++;
                    continue;
                }
                if (p_ < e_ && *p_ == ']') {
                    p_++;
                    return v;
                }
                fail("expected `,` or `]`");
            }
        }
        if (c == '"') {
            v.kind = JVal::Str;
            v.str = string();
            return v;
        }
        if (lit("true")) {
            v.kind = JVal::Bool;
            v.b = true;
            return v;
        }
        if (lit("false")) {
            v.kind = JVal::Bool;
            return v;
        }
        if (lit("null")) return v;
        if (c == '-' || (c >= '0' && c <= '9')) return number();
        fail("expected value");
    }
    static void utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (e_ - p_ < 4) fail("EOF while parsing a string");
        uint32_t v = 0;
        for (int i = 0; i < 4; i++) {
            char h = *p_++;
            v <<= 4;
            if (h >= '0' && h <= '9')
                v |= (uint32_t)(h - '0');
            else if (h >= 'a' && h <= 'f')
                v |= (uint32_t)(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F')
                v |= (uint32_t)(h - 'A' + 10);
            else
                fail("invalid escape");
        }
        return v;
    }
    std::string string() {
        p_++;  // opening quote
        std::string out;
        for (;;) {
            if (p_ == e_) fail("EOF while parsing a string");
            char c = *p_++;
            if (c == '"') return out;
            if ((unsigned char)c < 0x20) fail("control character while parsing a string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (p_ == e_) fail("EOF while parsing a string");
            char esc = *p_++;
            switch (esc) {
            case '"': out += '"'; break;
            case '\\': out += '\\'; break;
            case '/': out += '/'; break;
            case 'b': out += '\b'; break;
            case 'f': out += '\f'; break;
            case 'n': out += '\n'; break;
            case 'r': out += '\r'; break;
            case 't': out += '\t'; break;
            case 'u': {
                uint32_t cp = hex4();
                if (cp >= 0xD800 && cp < 0xDC00) {
                    if (!(e_ - p_ >= 2 && p_[0] == '\\' && p_[1] == 'u')) fail("lone leading surrogate in hex escape");
                    p_ += 2;
                    uint32_t lo = hex4();
                    if (lo < 0xDC00 || lo >= 0xE000) fail("lone leading surrogate in hex escape");
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                } else if (cp >= 0xDC00 && cp < 0xE000) {
                    fail("lone trailing surrogate in hex escape");
                }
                utf8(out, cp);
                break;
            }
            default: fail("invalid escape");
            }
        }
    }
    JVal number() {
        const char* s = p_;
        JVal v;
        v.kind = JVal::Num;
        v.integer = true;
        if (*p_ == '-') {
            v.negative = true;
            p_++;
        }
        if (p_ == e_ || !(*p_ >= '0' && *p_ <= '9')) fail("invalid number");
        if (*p_ == '0') {
            p_++;
        } else {
            while (p_ < e_ && *p_ >= '0' && *p_ <= '9') {
                uint64_t d = (uint64_t)(*p_ - '0');
                if (v.u > (UINT64_MAX - d) / 10) v.u_overflow = true;
                v.u = v.u * 10 + d;
                p_++;
            }
        }
        if (p_ < e_ && *p_ == '.') {
            v.integer = false;
            p_++;
            if (p_ == e_ || !(*p_ >= '0' && *p_ <= '9')) fail("invalid number");
            while (p_ < e_ && *p_ >= '0' && *p_ <= '9') p_++;
        }
        if (p_ < e_ && (*p_ == 'e' || *p_ == 'E')) {
            v.integer = false;
            p_++;
            if (p_ < e_ && (*p_ == '+' || *p_ == '-')) p_++;
            if (p_ == e_ || !(*p_ >= '0' && *p_ <= '9')) fail("invalid number");
            while (p_ < e_ && *p_ >= '0' && *p_ <= '9') p_++;
        }
        v.num = std::strtod(std::string(s, p_).c_str(), nullptr);
        return v;
    }
};

// ------------------------------------------------------------------ typed reads
// The reference's manifest structs (src/scene.rs:11-135).
struct Transform {
    float position[3], rotation[4], scale;
};
struct Geometry {
    std::string path;
    uint64_t vertex_offset, index_offset;
    uint32_t vertex_count, index_count;
};
struct Sdf {
    std::string path;
    uint64_t offset;
    uint32_t resolution;
    float bounds_min[3], bounds_max[3];
    bool conservative;
    std::string query;
    float error_bound;
};
struct Mesh {
    std::string id;
    Geometry geometry;
    Sdf sdf;
};
struct Material {
    std::string id;
    float base_color[4], roughness, metallic;
    std::string textures[4];  // base colour, roughness, metallic, normal
    bool has_texture[4] = {false, false, false, false};
    bool base_color_srgb = true;
    float normal_strength = 1.f;
    uint32_t texture_channels[4] = {0, 0, 0, 0};
};
struct Object {
    std::string id, mesh, material;
    Transform transform;
};
struct Light {
    std::string id, kind;
    float position[3], color[3], strength;
    float direction[3] = {0, 0, 0};
    float angle_radians = 0;
};
struct Camera {
    float position[3], rotation[4], fov_y_radians, near, far;
};
struct Manifest {
    uint32_t version;
    std::vector<Mesh> meshes;
    std::vector<Material> materials;
    std::vector<Object> objects;
    std::vector<Light> lights;
    Camera camera;
};

[[noreturn]] void err(const std::string& m) { throw Fail{m}; }

const JVal& field(const JVal& o, const char* k) {
    const JVal* v = o.get(k);
    if (!v) err(std::string("missing field `") + k + "`");
    return *v;
}
const JVal& as_obj(const JVal& v, const char* what) {
    if (v.kind != JVal::Obj) err(std::string("invalid type: expected struct ") + what);
    return v;
}
const JVal& as_arr(const JVal& v, const char* what) {
    if (v.kind != JVal::Arr) err(std::string("invalid type for `") + what + "`: expected a sequence");
    return v;
}
std::string rd_str(const JVal& o, const char* k) {
    const JVal& v = field(o, k);
    if (v.kind != JVal::Str) err(std::string("invalid type for `") + k + "`: expected a string");
    return v.str;
}
bool rd_bool(const JVal& v, const char* k) {
    if (v.kind != JVal::Bool) err(std::string("invalid type for `") + k + "`: expected a boolean");
    return v.b;
}
float num_f32(const JVal& v, const char* k) {
    if (v.kind != JVal::Num) err(std::string("invalid type for `") + k + "`: expected f32");
    return (float)v.num;
}
uint64_t num_uint(const JVal& v, const char* k, uint64_t max) {
    if (v.kind != JVal::Num || !v.integer || (v.negative && v.u != 0) || v.u_overflow || v.u > max)
        err(std::string("invalid value for `") + k + "`: expected an unsigned integer in range");
    return v.u;
}
float rd_f32(const JVal& o, const char* k) { return num_f32(field(o, k), k); }
void rd_vec(const JVal& v, const char* k, float* out, size_t n) {
    const JVal& a = as_arr(v, k);
    if (a.arr.size() != n) err(std::string("invalid length for `") + k + "`");
    for (size_t i = 0; i < n; i++) out[i] = num_f32(a.arr[i], k);
}

Transform read_transform(const JVal& v) {
    const JVal& o = as_obj(v, "Transform");
    for (const auto& kv : o.obj)
        if (kv.first != "position" && kv.first != "rotation" && kv.first != "scale")
            err("unknown field `" + kv.first + "`, expected one of `position`, `rotation`, `scale`");
    Transform t;
    rd_vec(field(o, "position"), "position", t.position, 3);
    rd_vec(field(o, "rotation"), "rotation", t.rotation, 4);
    t.scale = rd_f32(o, "scale");
    return t;
}

Manifest read_manifest(const JVal& root) {
    const JVal& r = as_obj(root, "Manifest");
    Manifest m;
    m.version = (uint32_t)num_uint(field(r, "version"), "version", UINT32_MAX);
    for (const JVal& jm : as_arr(field(r, "meshes"), "meshes").arr) {
        const JVal& o = as_obj(jm, "Mesh");
        Mesh x;
        x.id = rd_str(o, "id");
        const JVal& g = as_obj(field(o, "geometry"), "Geometry");
        x.geometry.path = rd_str(g, "path");
        x.geometry.vertex_offset = num_uint(field(g, "vertex_offset"), "vertex_offset", UINT64_MAX);
        x.geometry.vertex_count = (uint32_t)num_uint(field(g, "vertex_count"), "vertex_count", UINT32_MAX);
        x.geometry.index_offset = num_uint(field(g, "index_offset"), "index_offset", UINT64_MAX);
        x.geometry.index_count = (uint32_t)num_uint(field(g, "index_count"), "index_count", UINT32_MAX);
        const JVal& s = as_obj(field(o, "sdf"), "Sdf");
        x.sdf.path = rd_str(s, "path");
        x.sdf.offset = num_uint(field(s, "offset"), "offset", UINT64_MAX);
        x.sdf.resolution = (uint32_t)num_uint(field(s, "resolution"), "resolution", UINT32_MAX);
        rd_vec(field(s, "bounds_min"), "bounds_min", x.sdf.bounds_min, 3);
        rd_vec(field(s, "bounds_max"), "bounds_max", x.sdf.bounds_max, 3);
        x.sdf.conservative = rd_bool(field(s, "conservative"), "conservative");
        x.sdf.query = rd_str(s, "query");
        x.sdf.error_bound = rd_f32(s, "error_bound");
        m.meshes.push_back(std::move(x));
    }
    for (const JVal& jm : as_arr(field(r, "materials"), "materials").arr) {
        const JVal& o = as_obj(jm, "Material");
        Material x;
        x.id = rd_str(o, "id");
        rd_vec(field(o, "base_color"), "base_color", x.base_color, 4);
        x.roughness = rd_f32(o, "roughness");
        x.metallic = rd_f32(o, "metallic");
        const char* tex[4] = {"base_color_texture", "roughness_texture", "metallic_texture", "normal_texture"};
        for (int k = 0; k < 4; k++) {
            const JVal* t = o.get(tex[k]);
            if (!t || t->kind == JVal::Null) continue;
            if (t->kind != JVal::Str) err(std::string("invalid type for `") + tex[k] + "`: expected a string");
            x.textures[k] = t->str;
            x.has_texture[k] = true;
        }
        if (const JVal* v = o.get("base_color_srgb")) x.base_color_srgb = rd_bool(*v, "base_color_srgb");
        if (const JVal* v = o.get("normal_strength")) x.normal_strength = num_f32(*v, "normal_strength");
        if (const JVal* v = o.get("texture_channels")) {
            const JVal& a = as_arr(*v, "texture_channels");
            if (a.arr.size() != 4) err("invalid length for `texture_channels`");
            for (int k = 0; k < 4; k++) x.texture_channels[k] = (uint32_t)num_uint(a.arr[k], "texture_channels", UINT32_MAX);
        }
        m.materials.push_back(std::move(x));
    }
    for (const JVal& jo : as_arr(field(r, "objects"), "objects").arr) {
        const JVal& o = as_obj(jo, "Object");
        Object x;
        x.id = rd_str(o, "id");
        x.mesh = rd_str(o, "mesh");
        x.material = rd_str(o, "material");
        x.transform = read_transform(field(o, "transform"));
        m.objects.push_back(std::move(x));
    }
    for (const JVal& jl : as_arr(field(r, "lights"), "lights").arr) {
        const JVal& o = as_obj(jl, "Light");
        Light x;
        x.id = rd_str(o, "id");
        x.kind = rd_str(o, "type");
        rd_vec(field(o, "position"), "position", x.position, 3);
        rd_vec(field(o, "color"), "color", x.color, 3);
        x.strength = rd_f32(o, "strength");
        if (const JVal* v = o.get("direction")) rd_vec(*v, "direction", x.direction, 3);
        if (const JVal* v = o.get("angle_radians")) x.angle_radians = num_f32(*v, "angle_radians");
        m.lights.push_back(std::move(x));
    }
    const JVal& c = as_obj(field(r, "camera"), "Camera");
    rd_vec(field(c, "position"), "position", m.camera.position, 3);
    rd_vec(field(c, "rotation"), "rotation", m.camera.rotation, 4);
    m.camera.fov_y_radians = rd_f32(c, "fov_y_radians");
    m.camera.near = rd_f32(c, "near");
    m.camera.far = rd_f32(c, "far");
    return m;
}

// ------------------------------------------------------------------ validation
bool finite(const float* v, int n) {
    for (int i = 0; i < n; i++)
        if (!std::isfinite(v[i])) return false;
    return true;
}
float len2(const float* v, int n) {
    float s = 0.f;
    for (int i = 0; i < n; i++) s += v[i] * v[i];
    return s;
}
void ensure(bool ok, const std::string& m) {
    if (!ok) err(m);
}
std::string fmt_f(float v) {
    std::ostringstream os;
    os << v;
    return os.str();
}

std::string join(const std::string& root, const std::string& rel) {
    if (!rel.empty() && rel[0] == '/') return rel;
    if (root.empty()) return rel;
    return root + "/" + rel;
}
bool is_file(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0 && S_ISREG(st.st_mode);
}

void ids(const std::vector<const std::string*>& items, const char* kind) {
    std::set<std::string> seen;
    for (const std::string* id : items)
        ensure(!id->empty() && seen.insert(*id).second, std::string("duplicate/empty ") + kind + " ID: " + *id);
}

// Transform::validate (src/scene.rs:26-39).
void validate_transform(const Transform& t) {
    float q2 = len2(t.rotation, 4);
    ensure(finite(t.position, 3) && finite(t.rotation, 4) && std::isfinite(q2) && q2 > 1e-8f,
           "invalid position/quaternion");
    ensure(std::isfinite(t.scale) && t.scale > 1e-5f, "scale must be a positive finite uniform scalar");
}

// Scene::validate (src/scene.rs:256-382).
void validate(const Manifest& m, const std::string& root) {
    ensure(m.version == 1, "unsupported scene version " + std::to_string(m.version));
    std::vector<const std::string*> v;
    for (const Mesh& x : m.meshes) v.push_back(&x.id);
    ids(v, "mesh");
    v.clear();
    for (const Material& x : m.materials) v.push_back(&x.id);
    ids(v, "material");
    v.clear();
    for (const Object& x : m.objects) v.push_back(&x.id);
    for (const Light& x : m.lights) v.push_back(&x.id);
    ids(v, "object/light");
    ensure(!m.objects.empty(), "scene has no objects");
    for (const Mesh& mesh : m.meshes) {
        const Sdf& s = mesh.sdf;
        ensure(s.resolution >= 4 && s.resolution <= 256 && finite(s.bounds_min, 3) && finite(s.bounds_max, 3) &&
                   s.bounds_max[0] > s.bounds_min[0] && s.bounds_max[1] > s.bounds_min[1] &&
                   s.bounds_max[2] > s.bounds_min[2],
               "mesh " + mesh.id + ": invalid SDF bounds/resolution");
        ensure(s.conservative && s.query == "trilinear_bound" && std::isfinite(s.error_bound) && s.error_bound >= 0.f,
               "mesh " + mesh.id + ": SDF must be conservative with trilinear_bound query");
    }
    for (const Material& mat : m.materials) {
        bool ok = true;
        for (float c : mat.base_color) ok = ok && std::isfinite(c) && c >= 0.f;
        ensure(ok && std::isfinite(mat.roughness) && mat.roughness >= 0.f && mat.roughness <= 1.f &&
                   std::isfinite(mat.metallic) && mat.metallic >= 0.f && mat.metallic <= 1.f,
               "material " + mat.id + ": invalid PBR values");
        bool ch = true;
        for (uint32_t c : mat.texture_channels) ch = ch && c < 4;
        ensure(std::isfinite(mat.normal_strength) && mat.normal_strength >= 0.f && ch,
               "material " + mat.id + ": invalid texture settings");
        for (int k = 0; k < 4; k++) {
            if (!mat.has_texture[k]) continue;
            ensure(is_file(join(root, mat.textures[k])), "material " + mat.id + ": missing texture " + mat.textures[k]);
        }
    }
    for (const Object& obj : m.objects) {
        try {
            validate_transform(obj.transform);
        } catch (const Fail& f) {
            err("object " + obj.id + ": " + f.msg);
        }
        bool mesh = false, mat = false;
        for (const Mesh& x : m.meshes) mesh = mesh || x.id == obj.mesh;
        for (const Material& x : m.materials) mat = mat || x.id == obj.material;
        ensure(mesh, "object " + obj.id + ": missing mesh " + obj.mesh);
        ensure(mat, "object " + obj.id + ": missing material " + obj.material);
    }
    for (const Light& l : m.lights) {
        ensure(finite(l.position, 3) && finite(l.color, 3) &&
                   std::min(l.color[0], std::min(l.color[1], l.color[2])) >= 0.f && std::isfinite(l.strength) &&
                   l.strength >= 0.f,
               "light " + l.id + ": invalid values");
        if (l.kind == "point") continue;
        if (l.kind == "spot") {
            float d2 = len2(l.direction, 3);
            ensure(finite(l.direction, 3) && std::isfinite(d2) && d2 > 1e-8f && std::isfinite(l.angle_radians) &&
                       l.angle_radians > 0.f && l.angle_radians < (float)M_PI,
                   "light " + l.id + ": invalid spot cone/direction");
            continue;
        }
        err("light " + l.id + ": unsupported type " + l.kind);
    }
    const Camera& c = m.camera;
    float q2 = len2(c.rotation, 4);
    ensure(finite(c.position, 3) && finite(c.rotation, 4) && std::isfinite(q2) && q2 > 1e-8f && c.fov_y_radians > 0.f &&
               c.fov_y_radians < 3.13f && c.near > 0.f && std::isfinite(c.far) && c.far > c.near,
           "invalid camera");
}

// ------------------------------------------------------------------ binaries
struct Files {
    std::string root;
    std::map<std::string, std::shared_ptr<std::vector<uint8_t>>> cache;

    const std::vector<uint8_t>& read(const std::string& rel) {
        auto it = cache.find(rel);
        if (it != cache.end()) return *it->second;
        const std::string path = join(root, rel);
        std::ifstream f(path, std::ios::binary);
        if (!f) err(rel + ": " + std::strerror(errno));
        auto buf = std::make_shared<std::vector<uint8_t>>((std::istreambuf_iterator<char>(f)),
                                                          std::istreambuf_iterator<char>());
        if (f.bad()) err(rel + ": read error");
        cache[rel] = buf;
        return *buf;
    }
};

// range() of src/scene.rs:157-168: [offset, offset + count * stride) inside the file.
const uint8_t* range(const std::vector<uint8_t>& bytes, uint64_t offset, uint64_t count, uint64_t stride) {
    if (count != 0 && stride > UINT64_MAX / count) err("binary range overflow");
    const uint64_t n = count * stride;
    if (offset > UINT64_MAX - n) err("binary range overflow");
    const uint64_t end = offset + n;
    if (end > (uint64_t)bytes.size())
        err("binary range [" + std::to_string(offset) + "," + std::to_string(end) + ") exceeds " +
            std::to_string(bytes.size()) + " bytes");
    return bytes.data() + offset;
}

float le_f32(const uint8_t* p) {
    uint32_t u = (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
uint32_t le_u32(const uint8_t* p) {
    return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

struct MeshData {
    std::vector<irt_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<float> sdf;
};

// The per-mesh load of Scene::load (src/scene.rs:197-249).
MeshData load_mesh(Files& files, const Mesh& mesh) {
    MeshData d;
    const Geometry& g = mesh.geometry;
    const std::vector<uint8_t>& bytes = files.read(g.path);
    const uint8_t* vb = range(bytes, g.vertex_offset, g.vertex_count, 64);
    d.vertices.resize(g.vertex_count);
    for (uint32_t i = 0; i < g.vertex_count; i++) {
        float* dst = d.vertices[i].position;  // position, normal, tangent, uv: 16 consecutive f32
        for (int k = 0; k < 16; k++) dst[k] = le_f32(vb + (size_t)i * 64 + k * 4);
    }
    const uint8_t* ib = range(bytes, g.index_offset, g.index_count, 4);
    d.indices.resize(g.index_count);
    for (uint32_t i = 0; i < g.index_count; i++) d.indices[i] = le_u32(ib + (size_t)i * 4);
    ensure(g.vertex_count > 0 && g.index_count > 0 && g.index_count % 3 == 0, "geometry must have triangles");
    for (uint32_t j : d.indices) ensure(j < g.vertex_count, "index outside vertex range");
    for (const irt_vertex& v : d.vertices) ensure(finite(v.position, 16), "nonfinite vertex");
    const std::vector<uint8_t>& fb = files.read(mesh.sdf.path);
    const uint64_t r = mesh.sdf.resolution;
    const uint8_t* sb = range(fb, mesh.sdf.offset, r * r * r, 4);
    d.sdf.resize(r * r * r);
    for (size_t i = 0; i < d.sdf.size(); i++) d.sdf[i] = le_f32(sb + i * 4);
    for (float s : d.sdf) ensure(std::isfinite(s), "nonfinite SDF");
    return d;
}

void build(irt::Workload& w, const Manifest& m, std::vector<MeshData>& data) {
    using namespace irt;
    std::map<std::string, uint32_t> mesh_ids, material_ids;
    for (uint32_t i = 0; i < m.meshes.size(); i++) mesh_ids[m.meshes[i].id] = i;
    for (uint32_t i = 0; i < m.materials.size(); i++) material_ids[m.materials[i].id] = i;
    // Materials (src/renderer.rs:971-981).
    for (const Material& mat : m.materials) {
        irt_material g{};
        for (int k = 0; k < 4; k++) g.color[k] = mat.base_color[k];
        g.params[0] = mat.roughness;
        g.params[1] = mat.metallic;
        g.params[2] = mat.normal_strength;
        g.params[3] = mat.base_color_srgb ? 1.f : 0.f;
        for (int k = 0; k < 4; k++) {
            g.textures[k] = -1;
            g.channels[k] = mat.texture_channels[k];
        }
        w.materials.push_back(g);
    }
    // Lights (src/renderer.rs:1747-1755).
    for (const Light& l : m.lights) {
        irt_light g{};
        for (int k = 0; k < 3; k++) {
            g.position_strength[k] = l.position[k];
            g.direction_angle[k] = l.direction[k];
            g.color_type[k] = l.color[k];
        }
        g.position_strength[3] = l.strength;
        g.direction_angle[3] = l.angle_radians;
        g.color_type[3] = l.kind == "spot" ? 1.f : 0.f;
        w.lights.push_back(g);
    }
    // Objects in manifest order with Transform::matrix (src/scene.rs:18-25).
    for (const Object& o : m.objects) {
        Obj ob;
        ob.mesh = mesh_ids[o.mesh];
        ob.material = material_ids[o.material];
        double q[4] = {o.transform.rotation[0], o.transform.rotation[1], o.transform.rotation[2],
                       o.transform.rotation[3]};
        ob.model = scale_rotation_translation(o.transform.scale, q,
                                              D3{o.transform.position[0], o.transform.position[1],
                                                 o.transform.position[2]});
        ob.inv_model = inverse(ob.model);
        w.objs.push_back(ob);
    }
    // Meshes, atlas tiles of the largest resolution (src/renderer.rs:776-888).
    const uint32_t count = (uint32_t)m.meshes.size();
    uint32_t tile = 4;
    for (const Mesh& x : m.meshes) tile = std::max(tile, x.sdf.resolution);
    if (count == 0) tile = 4;
    irt_atlas_layout(std::max(count, 1u), tile, w.atlas_grid, w.atlas_dims);
    const size_t texels = (size_t)w.atlas_dims[0] * w.atlas_dims[1] * w.atlas_dims[2];
    if (w.spec.sdf_format == IRT_SDF_F16)
        w.atlas16.assign(texels, 0);
    else
        w.atlas32.assign(texels, 0.f);
    w.meshes.resize(count);
    w.mesh_desc.resize(count);
    // Meshes are independent (each fills its own atlas tile).  Host memory
    // exhaustion inside the parallel region is reported after it.
    bool oom = false;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t mi = 0; mi < (int64_t)count; mi++) try {
        const uint32_t i = (uint32_t)mi;
        const Mesh& x = m.meshes[i];
        MeshDesc& md = w.mesh_desc[i];
        md.triangles = true;
        md.resolution = x.sdf.resolution;
        for (int a = 0; a < 3; a++) {
            md.sdf_lo[a] = x.sdf.bounds_min[a];
            md.sdf_hi[a] = x.sdf.bounds_max[a];
        }
        md.vertices = std::move(data[i].vertices);
        md.indices = std::move(data[i].indices);
        build_tri_bvh(md.vertices.data(), md.indices.data(), (uint32_t)md.indices.size(), md.bvh);
        const uint32_t origin[3] = {(i % w.atlas_grid[0]) * tile, ((i / w.atlas_grid[0]) % w.atlas_grid[1]) * tile,
                                    (i / (w.atlas_grid[0] * w.atlas_grid[1])) * tile};
        irt_mesh_metadata(md.vertices.data(), (uint32_t)md.vertices.size(), md.indices.data(),
                          (uint32_t)md.indices.size(), data[i].sdf.data(), x.sdf.resolution, md.sdf_lo, md.sdf_hi,
                          origin, &w.meshes[i]);
        w.store_field(i, data[i].sdf.data(), x.sdf.resolution, origin);
        std::vector<float>().swap(data[i].sdf);
    } catch (const std::bad_alloc&) {
#pragma omp atomic write
        oom = true;
    }
    if (oom) throw std::bad_alloc();
    // Camera (src/scene.rs:110-128).
    w.loaded = true;
    for (int a = 0; a < 3; a++) w.cam_eye[a] = m.camera.position[a];
    for (int a = 0; a < 4; a++) w.cam_q[a] = m.camera.rotation[a];
    w.cam_fov = m.camera.fov_y_radians;
    w.cam_near = m.camera.near;
    w.cam_far = m.camera.far;
}

void put_error(char* out, uint64_t n, const std::string& m) {
    if (!out || n == 0) return;
    size_t k = std::min<size_t>((size_t)(n - 1), m.size());
    std::memcpy(out, m.data(), k);
    out[k] = '\0';
}

}  // namespace

extern "C" irt_status irt_workload_load(const char* manifest_path, const irt_workload_spec* spec, irt_workload** out,
                                        char* error, uint64_t error_len) {
    put_error(error, error_len, "");
    if (!manifest_path || !spec || !out) return IRT_E_INVALID;
    *out = nullptr;
    if (spec->width == 0 || spec->height == 0 || spec->width > 8192 || spec->height > 8192 || spec->vpl_count == 0 ||
        spec->vpl_bounces == 0 || (spec->sdf_format != IRT_SDF_F32 && spec->sdf_format != IRT_SDF_F16)) {
        put_error(error, error_len, "invalid workload spec");
        return IRT_E_INVALID;
    }
    const std::string path(manifest_path);
    std::string root;
    {
        size_t cut = path.find_last_of('/');
        root = cut == std::string::npos ? std::string() : path.substr(0, cut == 0 ? 1 : cut);
    }
    std::string stage = "reading " + path;
    try {
        std::ifstream f(path, std::ios::binary);
        if (!f) err(std::strerror(errno));
        std::string text((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        stage = "parsing " + path;
        Manifest m;
        {
            JVal doc = Parser(text.data(), text.size()).document();
            m = read_manifest(doc);
        }
        stage = "scene " + path;
        validate(m, root);
        Files files{root, {}};
        std::vector<MeshData> data;
        data.reserve(m.meshes.size());
        for (const Mesh& mesh : m.meshes) {
            stage = "mesh " + mesh.id;
            data.push_back(load_mesh(files, mesh));
        }
        files.cache.clear();
        stage = "scene " + path;
        for (const Material& mat : m.materials)
            for (bool t : mat.has_texture)
                ensure(!t, "material " + mat.id + ": textures are not supported by this loader");
        std::unique_ptr<irt_workload> wl(new (std::nothrow) irt_workload());
        if (!wl) {
            put_error(error, error_len, "out of host memory");
            return IRT_E_NOMEM;
        }
        wl->w.spec = *spec;
        build(wl->w, m, data);
        *out = wl.release();
        return IRT_OK;
    } catch (const Fail& e) {
        put_error(error, error_len, stage + ": " + e.msg);
        return IRT_E_INVALID;
    } catch (const std::bad_alloc&) {
        put_error(error, error_len, stage + ": out of host memory");
        return IRT_E_NOMEM;
    }
}
