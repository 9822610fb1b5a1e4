// scene_json.cpp — the reference JSON scene format read by the library itself, so that C and C++
// callers load a scene without Python (host code only, compiled with g++).
//
// Keys follow the reference SceneLoader (Utilities/SceneLoader.cpp:39-320): "Configuration"
// (timeStepSize, particleRadius, density0, viscosity, gravitation, cflMethod, cflFactor,
// cflMaxTimeStepSize, maxIterations, maxError, maxIterationsV, maxErrorV, enableDivergenceSolver),
// "FluidBlocks" (dense-mode boxes filled like DemoBase::createFluidBlocks,
// Demos/Common/DemoBase.cpp:539-603), "FluidModels" (partio .bgeo particle files with translation,
// rotationAxis / rotationAngle and scale, DemoBase::initFluidData :514-534) and "RigidBodies" (box
// walls sampled as a single-layer lattice of spacing 2r, or samples from a .bgeo "particleFile",
// Demos/StaticBoundaryDemo/main.cpp:416-420). Extension keys the reference does not read: "seed" and
// "jitter" (uniform jitter amplitude as a fraction of r), "precision" (32 / 64) and
// "learnedWarmStart". The arithmetic (in double, then rounded to float) and the jitter streams are
// those of the package's Python reader (splishsplash_for_cuda_b200/scene.py), so both readers give
// the same particles.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/dfsph_c.h"
#include "bgeo.h"

namespace dfsph {
void set_global_error(const std::string& msg);  // context.cu
}

namespace {

// ---- a small JSON reader (objects, arrays, numbers, strings, true / false / null) ---------------
struct JValue {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<JValue> arr;
    std::map<std::string, JValue> obj;
    const JValue* get(const char* key) const {
        if (kind != Object) return nullptr;
        auto it = obj.find(key);
        return it == obj.end() ? nullptr : &it->second;
    }
};

struct JParser {
    const std::string& s;
    size_t p = 0;
    std::string err;
    explicit JParser(const std::string& text) : s(text) {}
    void ws() {
        while (p < s.size() && (s[p] == ' ' || s[p] == '\t' || s[p] == '\n' || s[p] == '\r')) ++p;
    }
    bool fail(const std::string& m) {
        if (err.empty()) err = m + " at offset " + std::to_string(p);
        return false;
    }
    bool lit(const char* w) {
        const size_t n = std::strlen(w);
        if (s.compare(p, n, w) != 0) return fail(std::string("expected ") + w);
        p += n;
        return true;
    }
    bool string(std::string& out) {
        if (p >= s.size() || s[p] != '"') return fail("expected a string");
        ++p;
        out.clear();
        while (p < s.size() && s[p] != '"') {
            char c = s[p++];
            if (c == '\\') {
                if (p >= s.size()) return fail("bad escape");
                const char e = s[p++];
                switch (e) {
                    case '"': c = '"'; break;
                    case '\\': c = '\\'; break;
                    case '/': c = '/'; break;
                    case 'b': c = '\b'; break;
                    case 'f': c = '\f'; break;
                    case 'n': c = '\n'; break;
                    case 'r': c = '\r'; break;
                    case 't': c = '\t'; break;
                    case 'u': {
                        if (p + 4 > s.size()) return fail("bad \\u escape");
                        const unsigned v = (unsigned)std::stoul(s.substr(p, 4), nullptr, 16);
                        p += 4;
                        c = v < 128 ? (char)v : '?';  // scene keys and paths are ASCII
                        break;
                    }
                    default: return fail("bad escape");
                }
            }
            out.push_back(c);
        }
        if (p >= s.size()) return fail("unterminated string");
        ++p;
        return true;
    }
    bool value(JValue& v, int depth = 0) {
        if (depth > 64) return fail("nesting too deep");
        ws();
        if (p >= s.size()) return fail("unexpected end");
        const char c = s[p];
        if (c == '{') {
            ++p;
            v.kind = JValue::Object;
            ws();
            if (p < s.size() && s[p] == '}') return ++p, true;
            for (;;) {
                ws();
                std::string key;
                if (!string(key)) return false;
                ws();
                if (p >= s.size() || s[p] != ':') return fail("expected ':'");
                ++p;
                if (!value(v.obj[key], depth + 1)) return false;
                ws();
                if (p < s.size() && s[p] == ',') { ++p; continue; }
                if (p < s.size() && s[p] == '}') return ++p, true;
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            ++p;
            v.kind = JValue::Array;
            ws();
            if (p < s.size() && s[p] == ']') return ++p, true;
            for (;;) {
                v.arr.emplace_back();
                if (!value(v.arr.back(), depth + 1)) return false;
                ws();
                if (p < s.size() && s[p] == ',') { ++p; continue; }
                if (p < s.size() && s[p] == ']') return ++p, true;
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = JValue::String;
            return string(v.str);
        }
        if (c == 't') { v.kind = JValue::Bool; v.b = true; return lit("true"); }
        if (c == 'f') { v.kind = JValue::Bool; v.b = false; return lit("false"); }
        if (c == 'n') { v.kind = JValue::Null; return lit("null"); }
        const char* b = s.c_str() + p;
        char* e = nullptr;
        v.num = std::strtod(b, &e);
        if (e == b) return fail("bad value");
        v.kind = JValue::Number;
        p += (size_t)(e - b);
        return true;
    }
};

// ---- the Python reader's arithmetic ------------------------------------------------------------
// xoshiro256** (Blackman & Vigna) in 1024 interleaved streams, each seeded by four splitmix64
// steps from seed * 1024 + lane; value i comes from stream i % 1024 (scene.py xoshiro_uniform).
uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    uint64_t z = x;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
std::vector<double> xoshiro_uniform(size_t n, int64_t seed) {
    constexpr size_t kLanes = 1024;
    std::vector<double> out(n);
    if (!n) return out;
    std::vector<uint64_t> s0(kLanes), s1(kLanes), s2(kLanes), s3(kLanes);
    for (size_t l = 0; l < kLanes; ++l) {
        uint64_t x = ((uint64_t)seed & 0xFFFFFFFFFFFFull) * kLanes + l;
        uint64_t st[4];
        for (int k = 0; k < 4; ++k) {
            x += 0x9E3779B97F4A7C15ull;
            st[k] = splitmix64(x);
        }
        s0[l] = st[0]; s1[l] = st[1]; s2[l] = st[2]; s3[l] = st[3];
    }
    const size_t rounds = (n + kLanes - 1) / kLanes;
    for (size_t r = 0; r < rounds; ++r)
        for (size_t l = 0; l < kLanes; ++l) {
            const uint64_t v = rotl(s1[l] * 5, 7) * 9;
            const uint64_t t = s1[l] << 17;
            s2[l] ^= s0[l];
            s3[l] ^= s1[l];
            s1[l] ^= s2[l];
            s0[l] ^= s3[l];
            s2[l] ^= t;
            s3[l] = rotl(s3[l], 45);
            const size_t i = r * kLanes + l;
            if (i < n) out[i] = (double)(v >> 11) * (1.0 / 9007199254740992.0);
        }
    return out;
}

long round_half_even(double v) { return (long)std::nearbyint(v); }

// DemoBase::createFluidBlocks (dense mode): round(extent / 2r) - 1 particles per axis from min + 2r,
// x outer, y middle, z inner.
void fluid_block(const double mn[3], const double mx[3], double r, std::vector<double>& out) {
    const double d = 2.0 * r;
    long steps[3];
    for (int a = 0; a < 3; ++a) {
        steps[a] = round_half_even((mx[a] - mn[a]) / d) - 1;
        if (steps[a] < 0) steps[a] = 0;
    }
    for (long i = 0; i < steps[0]; ++i)
        for (long j = 0; j < steps[1]; ++j)
            for (long k = 0; k < steps[2]; ++k) {
                const long idx[3] = {i, j, k};
                for (int a = 0; a < 3; ++a) out.push_back((double)idx[a] * d + (mn[a] + d));
            }
}

// Single-layer lattice of spacing h on the surface of [mn, mx] (scene.py box_wall): faces
// perpendicular to x, then y, then z, each without the points the earlier faces produced.
void box_wall(const double mn[3], const double mx[3], double h, std::vector<double>& out) {
    long cnt[3];
    for (int a = 0; a < 3; ++a) cnt[a] = round_half_even((mx[a] - mn[a]) / h) + 1;
    for (int a = 0; a < 3; ++a) {
        int b = -1, c = -1;
        for (int d = 0; d < 3; ++d)
            if (d != a) (b < 0 ? b : c) = d;
        const long sides[2] = {0, cnt[a] - 1};
        for (long side : sides) {
            const long b0 = b < a ? 1 : 0, b1 = b < a ? cnt[b] - 1 : cnt[b];
            const long c0 = c < a ? 1 : 0, c1 = c < a ? cnt[c] - 1 : cnt[c];
            for (long ib = b0; ib < b1; ++ib)
                for (long ic = c0; ic < c1; ++ic) {
                    double idx[3];
                    idx[a] = (double)side;
                    idx[b] = (double)ib;
                    idx[c] = (double)ic;
                    for (int e = 0; e < 3; ++e) out.push_back(idx[e] * h + mn[e]);
                }
        }
    }
}

// Rotation of `angle` about `axis` (taken as given, as Eigen's AngleAxis in SceneLoader.cpp:228-233):
// R = cos(a) I + (1 - cos(a)) u u^T + sin(a) [u]x.
void angle_axis(const double u[3], double angle, double R[9]) {
    const double c = std::cos(angle), s = std::sin(angle);
    const double cross[9] = {0.0, -u[2], u[1], u[2], 0.0, -u[0], -u[1], u[0], 0.0};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[3 * i + j] = (i == j ? c : 0.0) + (1.0 - c) * u[i] * u[j] + s * cross[3 * i + j];
}

}  // namespace

struct dfsph_scene_file {
    dfsph_scene scene{};
    std::vector<float> fluid, fluid_vel, boundary;
    bool has_velocity = false;
    bool learned = false;
    std::map<std::string, double> learned_params;  // set_param keys
};

namespace {

bool readvec(const JValue* v, double out[3], std::string& err, const char* what) {
    if (!v) return true;
    if (v->kind != JValue::Array || v->arr.size() != 3) {
        err = std::string(what) + " must be an array of 3 numbers";
        return false;
    }
    for (int a = 0; a < 3; ++a) {
        if (v->arr[a].kind != JValue::Number) {
            err = std::string(what) + " must be an array of 3 numbers";
            return false;
        }
        out[a] = v->arr[a].num;
    }
    return true;
}

bool number(const JValue* v, double& out, std::string& err, const char* key) {
    if (!v) return true;
    if (v->kind == JValue::Number) out = v->num;
    else if (v->kind == JValue::Bool) out = v->b ? 1.0 : 0.0;
    else {
        err = std::string(key) + " must be a number";
        return false;
    }
    return true;
}

std::string dir_of(const std::string& path) {
    const size_t k = path.find_last_of('/');
    return k == std::string::npos ? std::string(".") : path.substr(0, k);
}
std::string relative(const std::string& scene_path, const std::string& file) {
    return (!file.empty() && file[0] == '/') ? file : dir_of(scene_path) + "/" + file;
}

// translation and rotationAxis / rotationAngle of a body or fluid model
void body_transform(const JValue& o, double t[3], double R[9], std::string& err, bool& ok) {
    t[0] = t[1] = t[2] = 0.0;
    for (int k = 0; k < 9; ++k) R[k] = (k % 4 == 0) ? 1.0 : 0.0;
    ok = readvec(o.get("translation"), t, err, "translation");
    const JValue* ax = o.get("rotationAxis");
    const JValue* an = o.get("rotationAngle");
    if (ok && ax && an && ax->kind != JValue::Null && an->kind != JValue::Null) {
        double u[3];
        double angle = 0.0;
        ok = readvec(ax, u, err, "rotationAxis") && number(an, angle, err, "rotationAngle");
        if (ok) angle_axis(u, angle, R);
    }
}

// x -> R (s x) + t for points of a particle file, in the Python reader's evaluation order
void place(const std::vector<float>& x, double s, const double R[9], const double t[3], std::vector<double>& out) {
    for (size_t i = 0; i + 2 < x.size(); i += 3) {
        const double p[3] = {(double)x[i] * s, (double)x[i + 1] * s, (double)x[i + 2] * s};
        for (int a = 0; a < 3; ++a) out.push_back((p[0] * R[3 * a] + p[1] * R[3 * a + 1] + p[2] * R[3 * a + 2]) + t[a]);
    }
}

int load(const char* path, dfsph_scene_file& f, std::string& err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        err = std::string("cannot open ") + path;
        return DFSPH_E_INVALID;
    }
    std::stringstream ss;
    ss << in.rdbuf();
    const std::string text = ss.str();
    JParser parser(text);
    JValue root;
    if (!parser.value(root)) {
        err = std::string(path) + ": " + parser.err;
        return DFSPH_E_INVALID;
    }
    if (root.kind != JValue::Object) {
        err = "a scene is a JSON object";
        return DFSPH_E_INVALID;
    }
    dfsph_scene& sc = f.scene;
    dfsph_scene_defaults(&sc);
    // SPH::TimeStep and SceneLoader defaults where the scene leaves a key out (scene.py Configuration)
    sc.time_step = 0.001;
    sc.particle_radius = 0.025;
    double seed = 1.0, jitter = 0.0, precision = 32.0;
    static const JValue empty{};
    const JValue* conf = root.get("Configuration");
    const JValue& c = conf ? *conf : empty;
    if (conf && conf->kind != JValue::Object) {
        err = "Configuration must be an object";
        return DFSPH_E_INVALID;
    }
    double v;
    struct Key {
        const char* name;
        double* dst;
    } keys[] = {{"timeStepSize", &sc.time_step}, {"particleRadius", &sc.particle_radius},
                {"density0", &sc.density0},       {"viscosity", &sc.viscosity},
                {"cflFactor", &sc.cfl_factor},    {"cflMaxTimeStepSize", &sc.cfl_max_time_step},
                {"maxError", &sc.max_error},      {"maxErrorV", &sc.max_error_v},
                {"seed", &seed},                  {"jitter", &jitter},
                {"precision", &precision}};
    for (const Key& k : keys)
        if (!number(c.get(k.name), *k.dst, err, k.name)) return DFSPH_E_INVALID;
    struct IKey {
        const char* name;
        int32_t* dst;
    } ikeys[] = {{"cflMethod", &sc.cfl_method},
                 {"maxIterations", &sc.max_iterations},
                 {"maxIterationsV", &sc.max_iterations_v},
                 {"enableDivergenceSolver", &sc.enable_divergence_solver}};
    for (const IKey& k : ikeys) {
        v = (double)*k.dst;
        if (!number(c.get(k.name), v, err, k.name)) return DFSPH_E_INVALID;
        *k.dst = (int32_t)v;
    }
    if (!readvec(c.get("gravitation"), sc.gravitation, err, "gravitation")) return DFSPH_E_INVALID;
    if (precision != 32.0 && precision != 64.0) {
        err = "precision must be 32 or 64";
        return DFSPH_E_INVALID;
    }
    sc.precision = (int32_t)precision;
    if (const JValue* l = c.get("learnedWarmStart")) {
        if (l->kind != JValue::Object) {
            err = "learnedWarmStart must be an object";
            return DFSPH_E_INVALID;
        }
        static const std::map<std::string, std::string> names = {
            {"enabled", ""}, {"trainInterval", "train_interval"}, {"trainIters", "train_iters"},
            {"trainBatch", "train_batch"}, {"learningRate", "learning_rate"}, {"damping", "warm_start_damping"},
            {"probe", "warm_start_probe"}};
        f.learned = true;
        for (const auto& kv : l->obj) {
            auto it = names.find(kv.first);
            if (it == names.end()) {
                err = "unknown learnedWarmStart key: " + kv.first;
                return DFSPH_E_INVALID;
            }
            double x = 0.0;
            if (!number(&kv.second, x, err, kv.first.c_str())) return DFSPH_E_INVALID;
            if (it->second.empty()) f.learned = x != 0.0;
            else f.learned_params[it->second] = x;
        }
    }
    const double r = sc.particle_radius;
    // fluid blocks, then the jitter of the blocks, then the particle files
    std::vector<double> fl;
    if (const JValue* blocks = root.get("FluidBlocks")) {
        for (const JValue& b : blocks->arr) {
            double start[3] = {0, 0, 0}, end[3] = {1, 1, 1}, scale[3] = {1, 1, 1}, trans[3] = {0, 0, 0}, dense = 0;
            if (!readvec(b.get("start"), start, err, "start") || !readvec(b.get("end"), end, err, "end") ||
                !readvec(b.get("scale"), scale, err, "scale") ||
                !readvec(b.get("translation"), trans, err, "translation") ||
                !number(b.get("denseMode"), dense, err, "denseMode"))
                return DFSPH_E_INVALID;
            if ((int)dense != 0) {
                err = "only denseMode 0 fluid blocks are supported";
                return DFSPH_E_INVALID;
            }
            double mn[3], mx[3];
            for (int a = 0; a < 3; ++a) {
                mn[a] = std::fmin(start[a], end[a]) * scale[a] + trans[a];
                mx[a] = std::fmax(start[a], end[a]) * scale[a] + trans[a];
            }
            fluid_block(mn, mx, r, fl);
        }
    }
    if (jitter != 0.0 && !fl.empty()) {
        const std::vector<double> u = xoshiro_uniform(fl.size(), (int64_t)seed);
        const double amp = jitter * r;
        for (size_t k = 0; k < fl.size(); ++k) fl[k] = fl[k] + (2.0 * u[k] - 1.0) * amp;
    }
    std::vector<double> flv(fl.size(), 0.0);
    if (const JValue* models = root.get("FluidModels")) {
        for (const JValue& m : models->arr) {
            const JValue* pf = m.get("particleFile");
            if (!pf) continue;
            std::vector<float> x, vx;
            bool hv = false;
            std::string berr;
            if (!dfsph::bgeo_read(relative(path, pf->str), x, vx, hv, berr)) {
                err = berr;
                return DFSPH_E_INVALID;
            }
            double t[3], R[9], s = 1.0;
            bool ok = true;
            body_transform(m, t, R, err, ok);
            if (!ok || !number(m.get("scale"), s, err, "scale")) return DFSPH_E_INVALID;
            place(x, s, R, t, fl);
            for (size_t k = 0; k < x.size(); ++k) flv.push_back(hv ? (double)vx[k] : 0.0);
            f.has_velocity = f.has_velocity || hv;
        }
    }
    std::vector<double> walls;
    if (const JValue* bodies = root.get("RigidBodies")) {
        for (const JValue& b : bodies->arr) {
            double scale[3] = {1, 1, 1}, trans[3] = {0, 0, 0};
            if (!readvec(b.get("scale"), scale, err, "scale") || !readvec(b.get("translation"), trans, err, "translation"))
                return DFSPH_E_INVALID;
            const JValue* pf = b.get("particleFile");
            if (pf && pf->kind == JValue::String && !pf->str.empty()) {
                std::vector<float> x, vx;
                bool hv = false;
                std::string berr;
                if (!dfsph::bgeo_read(relative(path, pf->str), x, vx, hv, berr)) {
                    err = berr;
                    return DFSPH_E_INVALID;
                }
                double t[3], R[9];
                bool ok = true;
                body_transform(b, t, R, err, ok);
                if (!ok) return DFSPH_E_INVALID;
                place(x, scale[0], R, t, walls);
                continue;
            }
            const JValue* geo = b.get("geometryFile");
            std::string g = geo && geo->kind == JValue::String ? geo->str : std::string();
            for (char& ch : g) ch = (char)std::tolower((unsigned char)ch);
            if (g.find("box") == std::string::npos) {
                err = "only box rigid bodies are supported, got '" + (geo ? geo->str : std::string()) + "'";
                return DFSPH_E_INVALID;
            }
            double mn[3], mx[3];
            for (int a = 0; a < 3; ++a) {
                mn[a] = trans[a] - 0.5 * scale[a];
                mx[a] = trans[a] + 0.5 * scale[a];
            }
            box_wall(mn, mx, 2.0 * r, walls);
        }
    }
    f.fluid.resize(fl.size());
    for (size_t k = 0; k < fl.size(); ++k) f.fluid[k] = (float)fl[k];
    f.fluid_vel.resize(flv.size());
    for (size_t k = 0; k < flv.size(); ++k) f.fluid_vel[k] = (float)flv[k];
    f.boundary.resize(walls.size());
    for (size_t k = 0; k < walls.size(); ++k) f.boundary[k] = (float)walls[k];
    sc.fluid_capacity = (uint32_t)std::max<size_t>(1, f.fluid.size() / 3);
    sc.boundary_capacity = (uint32_t)std::max<size_t>(1, f.boundary.size() / 3);
    return DFSPH_OK;
}

}  // namespace

extern "C" {

int dfsph_scene_load(const char* json_path, dfsph_scene* scene, dfsph_scene_file** out) {
    if (!json_path || !out) {
        dfsph::set_global_error("dfsph_scene_load: null argument");
        return DFSPH_E_INVALID;
    }
    *out = nullptr;
    auto f = std::make_unique<dfsph_scene_file>();
    std::string err;
    const int code = load(json_path, *f, err);
    if (code != DFSPH_OK) {
        dfsph::set_global_error(err);
        return code;
    }
    if (scene) *scene = f->scene;
    *out = f.release();
    return DFSPH_OK;
}

int dfsph_scene_file_counts(const dfsph_scene_file* f, uint32_t* n_fluid, uint32_t* n_boundary, int* has_velocity) {
    if (!f) {
        dfsph::set_global_error("null scene file");
        return DFSPH_E_INVALID;
    }
    if (n_fluid) *n_fluid = (uint32_t)(f->fluid.size() / 3);
    if (n_boundary) *n_boundary = (uint32_t)(f->boundary.size() / 3);
    if (has_velocity) *has_velocity = f->has_velocity ? 1 : 0;
    return DFSPH_OK;
}

int dfsph_scene_file_fluid(const dfsph_scene_file* f, float* xyz, float* vxyz) {
    if (!f) {
        dfsph::set_global_error("null scene file");
        return DFSPH_E_INVALID;
    }
    if (xyz && !f->fluid.empty()) std::memcpy(xyz, f->fluid.data(), f->fluid.size() * sizeof(float));
    if (vxyz && !f->fluid_vel.empty()) std::memcpy(vxyz, f->fluid_vel.data(), f->fluid_vel.size() * sizeof(float));
    return DFSPH_OK;
}

int dfsph_scene_file_boundary(const dfsph_scene_file* f, float* xyz) {
    if (!f) {
        dfsph::set_global_error("null scene file");
        return DFSPH_E_INVALID;
    }
    if (xyz && !f->boundary.empty()) std::memcpy(xyz, f->boundary.data(), f->boundary.size() * sizeof(float));
    return DFSPH_OK;
}

void dfsph_scene_file_free(dfsph_scene_file* f) { delete f; }

int dfsph_create_from_scene_file(const char* json_path, dfsph_ctx** out) {
    if (!out) {
        dfsph::set_global_error("null output");
        return DFSPH_E_INVALID;
    }
    *out = nullptr;
    dfsph_scene_file* f = nullptr;
    int code = dfsph_scene_load(json_path, nullptr, &f);
    if (code != DFSPH_OK) return code;
    std::unique_ptr<dfsph_scene_file> hold(f);
    dfsph_ctx* ctx = nullptr;
    code = dfsph_create(&f->scene, &ctx);
    if (code != DFSPH_OK) return code;
    const uint32_t n = (uint32_t)(f->fluid.size() / 3), nb = (uint32_t)(f->boundary.size() / 3);
    if (nb) code = dfsph_set_boundary(ctx, f->boundary.data(), nullptr, nb);
    if (code == DFSPH_OK)
        code = dfsph_upload_fluid(ctx, f->fluid.data(), f->has_velocity ? f->fluid_vel.data() : nullptr, nullptr, n);
    if (code == DFSPH_OK && f->learned) {  // its parameters first, then the mode (as the Python facade)
        for (const auto& kv : f->learned_params)
            if (code == DFSPH_OK) code = dfsph_set_param(ctx, kv.first.c_str(), kv.second);
        if (code == DFSPH_OK) code = dfsph_set_param(ctx, "learned_warm_start", 1.0);
    }
    if (code != DFSPH_OK) {
        const std::string msg = dfsph_last_error(ctx) ? dfsph_last_error(ctx) : "";
        dfsph_destroy(ctx);
        dfsph::set_global_error(msg);
        return code;
    }
    *out = ctx;
    return DFSPH_OK;
}

}  // extern "C"
