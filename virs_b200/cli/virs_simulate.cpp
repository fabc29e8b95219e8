// virs_simulate -- the command-line caller of libvirs_b200, in the form of
// the reference's `simulate` command (src/main.cpp:14-91):
//
//   virs_simulate simulate -i config.json [-o output_audio.wav]
//                 [--receiver X,Y,Z] [--steps N] [--storage f32|bf16|f16]
//
// The configuration is the reference's JSON file (Simulator::loadConfig,
// src/simulator/simulator.cpp:165-260): files.meshfile (the OBJ, opened
// relative to the working directory), files.audiofile (required, as there)
// and simulation.num_simulation_steps.  Three optional keys carry the
// material indexing and audio sources that the reference's TODO.md plans
// ("Material indexing", "Audio file implementation"):
//   "materials": [{"index": i, "type": "wall" | "source" | "ignore",
//                  "absorber": a}]   OBJ material i (the order of newmtl
//                                    declarations) and its role; default
//                                    the reference's: 0 wall, 1 source
//   "absorbers": [{"reflection": R, "cutoff": fc} | {"alpha": [a, b, c]}]
//                                    filter a: a first-order absorber or a
//                                    three-band cascade (FP64 designs);
//                                    default the reference's high-pass
//   "source": {"audio": true, "channel": k}
//                                    the speaker voxels play channel k of
//                                    files.audiofile (a WAV file) instead
//                                    of the reference's fixed pulse
//   "sources": [{"position": [x, y, z], "channel": k}]
//                                    point sources in metres (the voxel by
//                                    toVoxel and truncation, simulator.h:
//                                    32-45), each playing its channel of
//                                    files.audiofile, added to the field
// Then, as Simulator::simulate (simulator.cpp:933-1100): the mesh is voxelised and
// classified with the reference's defaults, the receiver is the voxel
// (334, 225, 270) unless --receiver names another, the steps run with the
// reference's RMS stop rule (here on the device), and the receiver trace is
// resampled to 48 kHz, peak-normalised and written as a 32-bit float mono
// WAV file ("output_audio.wav" unless -o names another).  The resampling is
// the library's (the reference's Chebyshev-I anti-alias design, then linear
// interpolation), not kfr's.
//
// Exit status: 0 on success, 2 for a usage or configuration error, 3 when
// the library reports an error (its message is printed).
#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "virs.hpp"

namespace {

// ---- a small JSON reader: objects, arrays, strings, numbers, literals ----------

struct Json {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    bool b = false;
    double num = 0;
    std::string str;
    std::vector<Json> arr;
    std::map<std::string, Json> obj;

    const Json *get(const std::string &k) const
    {
        if (kind != OBJ) return nullptr;
        auto it = obj.find(k);
        return it == obj.end() ? nullptr : &it->second;
    }
};

struct Parser {
    const std::string &s;
    size_t i = 0;
    std::string err;

    explicit Parser(const std::string &text) : s(text) {}

    void ws()
    {
        while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
    }
    bool fail(const std::string &m)
    {
        if (err.empty()) err = m + " at offset " + std::to_string(i);
        return false;
    }
    bool lit(const char *w)
    {
        const size_t n = std::strlen(w);
        if (s.compare(i, n, w) != 0) return fail(std::string("expected ") + w);
        i += n;
        return true;
    }
    bool string(std::string &out)
    {
        if (i >= s.size() || s[i] != '"') return fail("expected a string");
        ++i;
        out.clear();
        while (i < s.size() && s[i] != '"') {
            char c = s[i++];
            if (c == '\\') {
                if (i >= s.size()) return fail("unterminated escape");
                const char e = s[i++];
                switch (e) {
                case '"': case '\\': case '/': out += e; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    if (i + 4 > s.size()) return fail("short \\u escape");
                    const unsigned cp = (unsigned)std::strtoul(s.substr(i, 4).c_str(), nullptr, 16);
                    i += 4;
                    if (cp < 0x80) out += (char)cp;                 // paths and keys are ASCII here
                    else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
                    else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F));
                           out += (char)(0x80 | (cp & 0x3F)); }
                    break;
                }
                default: return fail("bad escape");
                }
            } else {
                out += c;
            }
        }
        if (i >= s.size()) return fail("unterminated string");
        ++i;
        return true;
    }
    bool value(Json &v, int depth = 0)
    {
        if (depth > 64) return fail("nesting too deep");
        ws();
        if (i >= s.size()) return fail("unexpected end");
        const char c = s[i];
        if (c == '{') {
            v.kind = Json::OBJ;
            ++i;
            ws();
            if (i < s.size() && s[i] == '}') { ++i; return true; }
            for (;;) {
                ws();
                std::string k;
                if (!string(k)) return false;
                ws();
                if (i >= s.size() || s[i] != ':') return fail("expected ':'");
                ++i;
                if (!value(v.obj[k], depth + 1)) return false;
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == '}') { ++i; return true; }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::ARR;
            ++i;
            ws();
            if (i < s.size() && s[i] == ']') { ++i; return true; }
            for (;;) {
                v.arr.emplace_back();
                if (!value(v.arr.back(), depth + 1)) return false;
                ws();
                if (i < s.size() && s[i] == ',') { ++i; continue; }
                if (i < s.size() && s[i] == ']') { ++i; return true; }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') { v.kind = Json::STR; return string(v.str); }
        if (c == 't') { v.kind = Json::BOOL; v.b = true; return lit("true"); }
        if (c == 'f') { v.kind = Json::BOOL; v.b = false; return lit("false"); }
        if (c == 'n') { v.kind = Json::NUL; return lit("null"); }
        char *end = nullptr;
        errno = 0;
        const double d = std::strtod(s.c_str() + i, &end);
        if (end == s.c_str() + i || errno) return fail("expected a value");
        v.kind = Json::NUM;
        v.num = d;
        i = (size_t)(end - s.c_str());
        return true;
    }
};

// ---- WAV input: one channel of PCM 16/24/32-bit or 32-bit float, as float -----

bool read_wav(const std::string &path, int channel, std::vector<float> &out, float &rate, std::string &err)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return false; }
    std::vector<unsigned char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    auto u16 = [&](size_t i) { return (uint32_t)b[i] | ((uint32_t)b[i + 1] << 8); };
    auto u32 = [&](size_t i) { return u16(i) | (u16(i + 2) << 16); };
    if (b.size() < 12 || std::memcmp(b.data(), "RIFF", 4) || std::memcmp(b.data() + 8, "WAVE", 4)) {
        err = path + ": not a RIFF/WAVE file";
        return false;
    }
    uint32_t fmt = 0, nch = 0, sr = 0, bits = 0;
    size_t data = 0, dlen = 0;
    for (size_t i = 12; i + 8 <= b.size();) {
        const uint32_t n = u32(i + 4);
        if (!std::memcmp(b.data() + i, "fmt ", 4) && n >= 16 && i + 8 + n <= b.size()) {
            fmt = u16(i + 8);
            nch = u16(i + 10);
            sr = u32(i + 12);
            bits = u16(i + 22);
            if (fmt == 0xFFFE && n >= 26) fmt = u16(i + 32); // WAVE_FORMAT_EXTENSIBLE: the sub-format
        } else if (!std::memcmp(b.data() + i, "data", 4)) {
            data = i + 8;
            dlen = std::min<size_t>(n, b.size() - data);
        }
        i += 8 + (size_t)n + (n & 1);
    }
    const bool ok = nch > 0 && sr > 0 && data &&
                    ((fmt == 1 && (bits == 16 || bits == 24 || bits == 32)) || (fmt == 3 && bits == 32));
    if (!ok) { err = path + ": unsupported WAV format (PCM 16/24/32-bit or 32-bit float)"; return false; }
    if (channel < 0 || (uint32_t)channel >= nch) {
        err = path + ": no channel " + std::to_string(channel) + " (" + std::to_string(nch) + " channels)";
        return false;
    }
    const size_t bps = bits / 8, frame = bps * nch, frames = dlen / frame;
    out.resize(frames);
    for (size_t k = 0; k < frames; ++k) {
        const unsigned char *p = b.data() + data + k * frame + (size_t)channel * bps;
        if (fmt == 3) {
            std::memcpy(&out[k], p, 4);
        } else if (bits == 16) {
            out[k] = (float)(int16_t)((uint16_t)p[0] | ((uint16_t)p[1] << 8)) / 32768.f;
        } else if (bits == 24) {
            int32_t v = (int32_t)((uint32_t)p[0] << 8 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 24) >> 8;
            out[k] = (float)v / 8388608.f;
        } else {
            int32_t v;
            std::memcpy(&v, p, 4);
            out[k] = (float)((double)v / 2147483648.0);
        }
    }
    rate = (float)sr;
    return true;
}

// ---- a 32-bit float mono WAV file (RIFF, format 3) -----------------------------

bool write_wav(const std::string &path, const std::vector<float> &x, uint32_t rate)
{
    std::ofstream f(path, std::ios::binary);
    if (!f) return false;
    auto u32 = [&](uint32_t v) { f.write(reinterpret_cast<const char *>(&v), 4); };
    auto u16 = [&](uint16_t v) { f.write(reinterpret_cast<const char *>(&v), 2); };
    const uint32_t data = (uint32_t)(x.size() * 4);
    f.write("RIFF", 4);
    u32(4 + 26 + 12 + 8 + data);
    f.write("WAVE", 4);
    f.write("fmt ", 4);
    u32(18);
    u16(3);            // IEEE float
    u16(1);            // mono
    u32(rate);
    u32(rate * 4);
    u16(4);
    u16(32);
    u16(0);            // no extension
    f.write("fact", 4);
    u32(4);
    u32((uint32_t)x.size());
    f.write("data", 4);
    u32(data);
    f.write(reinterpret_cast<const char *>(x.data()), data);
    return (bool)f;
}

int usage(const char *msg)
{
    if (msg) std::fprintf(stderr, "virs_simulate: %s\n", msg);
    std::fprintf(stderr,
                 "usage: virs_simulate simulate -i CONFIG.json [-o OUTPUT.wav] [--receiver X,Y,Z] [--steps N]\n"
                 "                    [--storage f32|bf16|f16]\n"
                 "Runs the simulation described by the reference's JSON configuration on the GPU and writes\n"
                 "the receiver's impulse response at 48 kHz as a 32-bit float mono WAV file.\n");
    return msg ? 2 : 0;
}

} // namespace

int main(int argc, char **argv)
{
    std::string cmd, input, output = "output_audio.wav", storage = "f32";
    long long rx = 334, ry = 225, rz = 270; // the reference's receiver voxel (simulator_gpu.cu:295-300)
    long long steps_override = -1;
    for (int k = 1; k < argc; ++k) {
        const std::string a = argv[k];
        auto next = [&](const char *what) -> const char * {
            if (k + 1 >= argc) return nullptr;
            (void)what;
            return argv[++k];
        };
        if (a == "-h" || a == "--help") return usage(nullptr);
        if (a == "-i" || a == "--input") {
            const char *v = next("input");
            if (!v) return usage("-i needs a file name");
            input = v;
        } else if (a == "-o" || a == "--output") {
            const char *v = next("output");
            if (!v) return usage("-o needs a file name");
            output = v;
        } else if (a == "--receiver") {
            const char *v = next("receiver");
            if (!v || std::sscanf(v, "%lld,%lld,%lld", &rx, &ry, &rz) != 3) return usage("--receiver needs X,Y,Z");
        } else if (a == "--steps") {
            const char *v = next("steps");
            if (!v || std::sscanf(v, "%lld", &steps_override) != 1 || steps_override < 1)
                return usage("--steps needs a positive count");
        } else if (a == "--storage") {
            const char *v = next("storage");
            if (!v) return usage("--storage needs f32, bf16 or f16");
            storage = v;
        } else if (cmd.empty() && a[0] != '-') {
            cmd = a;
        } else {
            return usage(("unknown argument " + a).c_str());
        }
    }
    if (cmd != "simulate") return usage(cmd.empty() ? "missing command (simulate)" : "only the simulate command exists");
    if (input.empty()) return usage("missing -i CONFIG.json");
    if (storage != "f32" && storage != "bf16" && storage != "f16") return usage("--storage must be f32, bf16 or f16");

    // the configuration, with the reference's required keys
    std::ifstream cf(input);
    if (!cf) return usage(("cannot open " + input).c_str());
    std::stringstream ss;
    ss << cf.rdbuf();
    const std::string text = ss.str();
    Json cfg;
    Parser ps(text);
    if (!ps.value(cfg)) return usage((input + ": " + ps.err).c_str());
    const Json *files = cfg.get("files");
    if (!files) return usage("configuration has no 'files' key");
    const Json *mesh = files->get("meshfile");
    if (!mesh || mesh->kind != Json::STR || mesh->str.empty()) return usage("configuration has no 'meshfile' key");
    const Json *audio = files->get("audiofile");
    if (!audio || audio->kind != Json::STR || audio->str.empty()) return usage("configuration has no 'audiofile' key");
    const Json *sim_cfg = cfg.get("simulation");
    if (!sim_cfg) return usage("configuration has no 'simulation' key");
    const Json *nsteps = sim_cfg->get("num_simulation_steps");
    if (!nsteps || nsteps->kind != Json::NUM || nsteps->num < 1 || nsteps->num != std::floor(nsteps->num))
        return usage("configuration has no positive integer 'num_simulation_steps'");
    const uint64_t steps = steps_override > 0 ? (uint64_t)steps_override : (uint64_t)nsteps->num;

    // material indexing: OBJ material id -> role (virs_set_material_roles)
    std::vector<uint8_t> roles;
    uint32_t max_absorber = 0;
    bool any_wall_role = false;
    if (const Json *mats = cfg.get("materials")) {
        if (mats->kind != Json::ARR) return usage("'materials' must be an array");
        for (const Json &m : mats->arr) {
            const Json *ix = m.get("index"), *ty = m.get("type");
            if (!ix || ix->kind != Json::NUM || ix->num < 0 || ix->num > 255 || ix->num != std::floor(ix->num))
                return usage("each material needs an integer 'index' in 0..255");
            if (!ty || ty->kind != Json::STR) return usage("each material needs a 'type' (wall, source or ignore)");
            const size_t i = (size_t)ix->num;
            if (roles.size() <= i) roles.resize(i + 1, VIRS_ROLE_IGNORE);
            if (ty->str == "wall") {
                const Json *ab = m.get("absorber");
                double a = 0;
                if (ab) {
                    if (ab->kind != Json::NUM || ab->num < 0 || ab->num > 63 || ab->num != std::floor(ab->num))
                        return usage("a wall's 'absorber' must be an integer in 0..63");
                    a = ab->num;
                }
                roles[i] = (uint8_t)a;
                max_absorber = std::max(max_absorber, (uint32_t)a);
                any_wall_role = true;
            } else if (ty->str == "source") {
                roles[i] = VIRS_ROLE_SOURCE;
            } else if (ty->str == "ignore") {
                roles[i] = VIRS_ROLE_IGNORE;
            } else {
                return usage(("unknown material type '" + ty->str + "'").c_str());
            }
        }
    }
    // absorbers: one filter cascade per absorber index
    const Json *absorbers = cfg.get("absorbers");
    if (absorbers && (absorbers->kind != Json::ARR || absorbers->arr.empty()))
        return usage("'absorbers' must be a non-empty array");
    if (absorbers && any_wall_role && max_absorber >= absorbers->arr.size())
        return usage("a material names an absorber that 'absorbers' does not define");
    if (!absorbers && any_wall_role && max_absorber > 0)
        return usage("materials name absorbers beyond 0 but 'absorbers' is missing");
    if (absorbers)
        for (const Json &a : absorbers->arr) {
            const Json *r = a.get("reflection"), *fc = a.get("cutoff"), *al = a.get("alpha");
            const bool first = r && fc && r->kind == Json::NUM && fc->kind == Json::NUM;
            const bool bands = al && al->kind == Json::ARR && al->arr.size() == 3;
            if (first == bands) return usage("each absorber is {reflection, cutoff} or {alpha: [3 values]}");
            if (bands)
                for (const Json &v : al->arr)
                    if (v.kind != Json::NUM) return usage("'alpha' values must be numbers");
        }
    // the speaker voxels: the reference's pulse, or a channel of the audio file
    int audio_channel = -1;
    if (const Json *src = cfg.get("source")) {
        const Json *au = src->get("audio"), *ch = src->get("channel");
        if (au && au->kind == Json::BOOL && au->b) {
            audio_channel = 0;
            if (ch) {
                if (ch->kind != Json::NUM || ch->num < 0 || ch->num != std::floor(ch->num))
                    return usage("'channel' must be a non-negative integer");
                audio_channel = (int)ch->num;
            }
        }
    }
    std::vector<float> audio_samples;
    float audio_rate = 0.f;
    if (audio_channel >= 0) {
        std::string err;
        if (!read_wav(audio->str, audio_channel, audio_samples, audio_rate, err)) return usage(err.c_str());
        if (audio_samples.empty()) return usage("the audio file has no samples");
    }
    // point sources playing channels of the audio file
    struct PointSource {
        float pos[3];
        std::vector<float> samples;
    };
    std::vector<PointSource> points;
    float points_rate = 0.f;
    if (const Json *ps = cfg.get("sources")) {
        if (ps->kind != Json::ARR) return usage("'sources' must be an array");
        for (const Json &e : ps->arr) {
            const Json *pos = e.get("position"), *ch = e.get("channel");
            if (!pos || pos->kind != Json::ARR || pos->arr.size() != 3 || pos->arr[0].kind != Json::NUM ||
                pos->arr[1].kind != Json::NUM || pos->arr[2].kind != Json::NUM)
                return usage("each source needs a 'position' [x, y, z] in metres");
            int c = 0;
            if (ch) {
                if (ch->kind != Json::NUM || ch->num < 0 || ch->num != std::floor(ch->num))
                    return usage("a source's 'channel' must be a non-negative integer");
                c = (int)ch->num;
            }
            PointSource p;
            for (int k = 0; k < 3; ++k) p.pos[k] = (float)pos->arr[k].num;
            std::string err;
            if (!read_wav(audio->str, c, p.samples, points_rate, err)) return usage(err.c_str());
            if (p.samples.empty()) return usage("the audio file has no samples");
            points.push_back(std::move(p));
        }
    }

    try {
        virs_params p = virs::default_params();
        p.storage = storage == "bf16" ? VIRS_STORAGE_BF16 : storage == "f16" ? VIRS_STORAGE_F16 : VIRS_STORAGE_F32;
        virs::Simulator sim(p);
        if (!roles.empty()) sim.set_material_roles(roles);
        sim.load_obj(mesh->str);
        sim.classify();
        const virs_grid_info g = sim.info();
        if (absorbers) {
            // FP64 designs at the simulation rate; shorter cascades padded
            // with pass-through sections {1, 0, 0, 0, 0}
            std::vector<std::vector<double>> des;
            uint32_t ns = 1;
            for (const Json &a : absorbers->arr) {
                std::vector<double> c;
                if (const Json *al = a.get("alpha")) {
                    const double alpha[3] = {al->arr[0].num, al->arr[1].num, al->arr[2].num};
                    c.resize(15);
                    virs::check(virs_design_octave_cascade(g.sample_rate, alpha, nullptr, c.data()));
                } else {
                    c.resize(5);
                    virs::check(virs_design_first_order(g.sample_rate, a.get("reflection")->num, a.get("cutoff")->num,
                                                        c.data()));
                }
                ns = std::max<uint32_t>(ns, (uint32_t)(c.size() / 5));
                des.push_back(std::move(c));
            }
            std::vector<float> coef;
            for (const auto &c : des)
                for (uint32_t q = 0; q < ns; ++q)
                    for (int k = 0; k < 5; ++k)
                        coef.push_back(q * 5 < c.size() ? (float)c[q * 5 + k] : (k == 0 ? 1.f : 0.f));
            sim.set_filters((uint32_t)des.size(), ns, coef);
        }
        if (audio_channel >= 0)
            virs::check(virs_set_hard_source_audio(sim.handle(), audio_samples.data(), audio_samples.size(), audio_rate,
                                                   steps));
        if (!points.empty()) {
            // toVoxel, then truncation (Simulator::getGridIdxFromVecPos)
            std::vector<uint64_t> idx;
            const size_t len = points[0].samples.size(); // every channel of one file has the same length
            std::vector<float> chans;
            for (const PointSource &p : points) {
                uint64_t v[3];
                const uint64_t dim[3] = {g.nx, g.ny, g.nz};
                for (int k = 0; k < 3; ++k) {
                    const float t = (p.pos[k] - g.bbox_min[k]) / g.cell_size;
                    if (!(t >= 0.f) || (uint64_t)t >= dim[k]) {
                        std::fprintf(stderr, "virs_simulate: source at (%g, %g, %g) m is outside the grid\n",
                                     (double)p.pos[0], (double)p.pos[1], (double)p.pos[2]);
                        return 2;
                    }
                    v[k] = (uint64_t)t;
                }
                idx.push_back((v[2] * g.ny + v[1]) * g.nx + v[0]);
                chans.insert(chans.end(), p.samples.begin(), p.samples.end());
            }
            virs::check(virs_set_sources_audio(sim.handle(), (uint32_t)idx.size(), idx.data(), chans.data(), len,
                                               points_rate, steps));
        }
        if (rx < 0 || ry < 0 || rz < 0 || (uint64_t)rx >= g.nx || (uint64_t)ry >= g.ny || (uint64_t)rz >= g.nz) {
            std::fprintf(stderr, "virs_simulate: receiver (%lld, %lld, %lld) is outside the %llux%llux%llu grid; "
                                 "pass --receiver X,Y,Z\n",
                         rx, ry, rz, (unsigned long long)g.nx, (unsigned long long)g.ny, (unsigned long long)g.nz);
            return 2;
        }
        sim.set_receivers({((uint64_t)rz * g.ny + (uint64_t)ry) * g.nx + (uint64_t)rx});
        virs::check(virs_set_stop_rule(sim.handle(), 1));
        sim.start(steps);
        sim.autotune(); // tiling and steps per pass for this grid; results are the same bits either way
        sim.run(steps);
        sim.synchronize();
        const virs_grid_info after = sim.info();
        int stopped = 0;
        uint64_t stop_step = 0;
        virs::check(virs_get_stop(sim.handle(), &stopped, &stop_step));

        // 48 kHz: the reference's anti-alias design, linear interpolation, peak normalisation
        const double rate = 48000.0;
        double sos[32 * 6];
        uint32_t ns = 0;
        virs::check(virs_design_chebyshev_lowpass(g.sample_rate, 0.45 * rate, 0.5 * rate, 0.5, 90.0, sos, 32, &ns));
        uint64_t n = 0;
        virs::check(virs_postprocess_ir(sim.handle(), rate, sos, ns, 1, nullptr, 0, &n));
        std::vector<float> wav((size_t)n);
        virs::check(virs_postprocess_ir(sim.handle(), rate, sos, ns, 1, wav.data(), wav.size(), &n));
        if (!write_wav(output, wav, (uint32_t)rate)) {
            std::fprintf(stderr, "virs_simulate: cannot write %s\n", output.c_str());
            return 2;
        }
        std::printf("grid %llux%llux%llu, h %.6g m, %llu boundary voxels\n", (unsigned long long)g.nx,
                    (unsigned long long)g.ny, (unsigned long long)g.nz, (double)g.cell_size,
                    (unsigned long long)g.boundary_count);
        if (stopped)
            std::printf("stopped by the RMS rule after step %llu of %llu\n", (unsigned long long)stop_step,
                        (unsigned long long)steps);
        std::printf("%llu steps, %llu samples at 48 kHz written to %s\n", (unsigned long long)after.steps_done,
                    (unsigned long long)n, output.c_str());
    } catch (const virs::Error &e) {
        std::fprintf(stderr, "virs_simulate: %s\n", e.what());
        return 3;
    }
    return 0;
}
