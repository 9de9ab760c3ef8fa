// Launch-shape autotuner for sm_100a: the analogue of the reference's FFTW
// planning with MEASURE and its wisdom files (src/fft/transforms.cpp:190-278,
// src/fft/wisdom.cpp:11-32).
//
// For each mesh, the first FP64 context times on its own device buffers, with
// CUDA events on its stream (a mixed-precision context times the x-stage and
// Chebyshev forms on its FP32 buffers, under a key of its own),
//   - the kx lines per block of the z transforms (8..17): the z synthesis of
//     the six nonlinear-term fields plus the z analysis of three, and
//   - the form of the register-form x stage: 2 or 4 rows per block, 4 rows
//     with the forward phases split over lane pairs, or a half-warp per row pair,
//   - the Chebyshev synthesis (six fields) and analysis (three fields) in the
//     matrix form (FP64 MMA products) and in the FFT form (DCT-I through one
//     length-NY2 FFT per column; meshes whose NY2 has a register split),
// keeps the fastest of each, and caches the choice for the process under a key
// of the mesh and the device.  cdns_wisdom_export / cdns_wisdom_import write
// and read that cache as JSON so that later processes skip the timing.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "context.cuh"

namespace cdns {

namespace {

struct Choice {
    int ztl = 0;     // 0: the padding rule
    int yform = 0;   // bit 0 synthesis, bit 1 analysis in the FFT form
    int xrw = 0;     // rows per block of the register-form x stage (0: 4)
};

std::mutex g_mu;
std::map<std::string, Choice> g_wisdom;
std::once_flag g_env_import;

std::string mesh_key(const cdns_ctx *c) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, c->device);
    const Dims &d = c->d;
    // the device name holds at most 256 characters; seven ints and separators follow
    char buf[256 + 96];
    std::snprintf(buf, sizeof buf, "%.256s/%d|%d,%d,%d|%d,%d,%d%s", prop.name, prop.multiProcessorCount, d.NX2,
                  d.NY2, d.NZ2, d.NXS, d.NYS, d.NZS, c->mixed ? "|fp32" : "");
    return buf;
}

// Best (minimum) of `reps` timed runs of fn on the context stream, in ms.
template <typename Fn> int time_min(cdns_ctx *c, int reps, Fn fn, float &best) {
    cudaEvent_t a, b;
    CK(cudaEventCreate(&a));
    CK(cudaEventCreate(&b));
    best = 1e30f;
    fn();   // warm-up
    for (int r = 0; r < reps; ++r) {
        CK(cudaEventRecord(a, c->stream));
        fn();
        CK(cudaEventRecord(b, c->stream));
        CK(cudaEventSynchronize(b));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        if (ms < best) best = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CK(cudaGetLastError());
    return CDNS_OK;
}

// FP32 stage buffers (mixed form): the forms of the x stage and of the
// Chebyshev transforms are timed on the context's FP32 buffers; the z
// transforms keep their rule.
int measure_fp32(cdns_ctx *c, Choice &out) {
    const Dims d = c->d;
    cudaStream_t s = c->stream;
    const int reps = 3;
    out = Choice{};
    {
        float2 *G = reinterpret_cast<float2 *>(c->G), *H = reinterpret_cast<float2 *>(c->H);
        float best_x = 1e30f;
        for (int rw : {4, 2, 1, 3, 5}) {
            Dims dx = d;
            dx.xrw = rw;
            float ms;
            int r = time_min(c, reps, [&] { launch_x_cross(dx, c->t.root_x, G, H, c->mean, s); }, ms);
            if (r) return r;
            if (ms < best_x) {
                best_x = ms;
                out.xrw = rw;
            }
        }
    }
    if (!ydct_available(d, c->t)) return CDNS_OK;
    float2 *F = reinterpret_cast<float2 *>(c->F);
    Tables t = c->t;
    float m_syn, f_syn, m_ana, f_ana;
    int r = 0;
    t.yform = 0;
    if ((r = time_min(c, reps, [&] { launch_ysynth(d, t, c->U[0], c->om, 3, 6, F, c->mean, s); }, m_syn))) return r;
    if ((r = time_min(c, reps, [&] { launch_yanalysis(d, t, F, c->aux, 3, s); }, m_ana))) return r;
    t.yform = 3;
    if ((r = time_min(c, reps, [&] { launch_ysynth(d, t, c->U[0], c->om, 3, 6, F, c->mean, s); }, f_syn))) return r;
    if ((r = time_min(c, reps, [&] { launch_yanalysis(d, t, F, c->aux, 3, s); }, f_ana))) return r;
    out.yform = (f_syn < m_syn ? 1 : 0) | (f_ana < m_ana ? 2 : 0);
    return CDNS_OK;
}

int measure(cdns_ctx *c, Choice &out) {
    if (c->mixed) return measure_fp32(c, out);
    const Dims base = c->d;
    cudaStream_t s = c->stream;
    const int reps = 3;
    // z transforms: 6 fields backward + 3 forward, as in the step
    float best = 1e30f;
    int best_tl = 0;
    for (int tl = 8; tl <= 17; ++tl) {
        Dims d = base;
        d.ztl = tl;
        float ms;
        int r = time_min(c, reps, [&] {
            launch_z_backward(d, c->pz, c->t.root_z, c->F, c->G, 6, s);
            launch_z_forward(d, c->pz, c->t.root_z, c->H, c->F, 3, s);
        }, ms);
        if (r) return r;
        if (ms < best) {
            best = ms;
            best_tl = tl;
        }
    }
    out.ztl = best_tl;
    Dims d = base;
    d.ztl = best_tl;
    // x stage: 2 or 4 rows per block (smaller blocks couple fewer warps at each
    // barrier) or the half-warp form (1: a half-warp per row pair, no block barrier)
    {
        float best_x = 1e30f;
        for (int rw : {4, 2, 1, 3, 5}) {
            Dims dx = d;
            dx.xrw = rw;
            float ms;
            int r = time_min(c, reps, [&] { launch_x_cross(dx, c->px, c->t.root_x, c->G, c->H, s); }, ms);
            if (r) return r;
            if (ms < best_x) {
                best_x = ms;
                out.xrw = rw;
            }
        }
    }
    out.yform = 0;
    if (ydct_available(d, c->t)) {
        Tables t = c->t;
        float m_syn, f_syn, m_ana, f_ana;
        int r = 0;
        t.yform = 0;
        if ((r = time_min(c, reps, [&] { launch_ysynth(d, t, c->U[0], c->om, 3, 6, c->F, s); }, m_syn))) return r;
        if ((r = time_min(c, reps, [&] { launch_yanalysis(d, t, c->F, c->aux, 3, s); }, m_ana))) return r;
        t.yform = 3;
        if ((r = time_min(c, reps, [&] { launch_ysynth(d, t, c->U[0], c->om, 3, 6, c->F, s); }, f_syn))) return r;
        if ((r = time_min(c, reps, [&] { launch_yanalysis(d, t, c->F, c->aux, 3, s); }, f_ana))) return r;
        out.yform = (f_syn < m_syn ? 1 : 0) | (f_ana < m_ana ? 2 : 0);
    }
    return CDNS_OK;
}

// CDNS_X_STAGE=rows4|rows2|halfwarp|split fixes the form of the register-form x
// stage (comparisons, tests); FP32 contexts honour it too.
void apply_x_stage_env(cdns_ctx *c) {
    if (const char *e = std::getenv("CDNS_X_STAGE")) {
        if (std::strcmp(e, "rows4") == 0) c->d.xrw = 4;
        else if (std::strcmp(e, "rows2") == 0) c->d.xrw = 2;
        else if (std::strcmp(e, "halfwarp") == 0) c->d.xrw = 1;
        else if (std::strcmp(e, "split") == 0) c->d.xrw = 3;
        else if (std::strcmp(e, "split2") == 0) c->d.xrw = 5;
    }
}

void apply(cdns_ctx *c, const Choice &ch) {
    c->d.ztl = ch.ztl;
    c->d.xrw = ch.xrw;
    c->t.yform = ch.yform;
    // CDNS_Y_TRANSFORM=matrix|fft fixes the Chebyshev form (comparisons, tests)
    if (const char *e = std::getenv("CDNS_Y_TRANSFORM")) {
        if (std::strcmp(e, "matrix") == 0) c->t.yform = 0;
        else if (std::strcmp(e, "fft") == 0) c->t.yform = 3;
    }
    apply_x_stage_env(c);
}

}  // namespace
}  // namespace cdns

extern "C" int cdns_wisdom_import(const char *path);
extern "C" int cdns_wisdom_export(const char *path);

namespace cdns {

// Picks the launch shapes of an FP64 context: from the process cache or the
// wisdom, else by timing (unless CDNS_TUNE=0, which keeps the fixed rules).
// CDNS_WISDOM=<file> imports that file once per process (if it exists) and
// exports the cache to it after every new measurement, so that a later run --
// a profiled one, whose timings would mislead the tuner -- reuses the choices.
int tune_context(cdns_ctx *c, bool force) {
    if (c->pen) {
        // a pencil rank holds part of the mesh: timing it would file its
        // shapes under the whole mesh's key, so it keeps the rule-based ones
        apply(c, Choice{});
        return CDNS_OK;
    }
    const char *wfile = std::getenv("CDNS_WISDOM");
    if (wfile && *wfile) {
        std::call_once(g_env_import, [&] {
            if (std::FILE *f = std::fopen(wfile, "r")) {
                std::fclose(f);
                cdns_wisdom_import(wfile);   // a malformed file leaves the cache as it is
            }
        });
    }
    const std::string key = mesh_key(c);
    Choice ch;
    bool have = false;
    if (!force) {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_wisdom.find(key);
        if (it != g_wisdom.end()) {
            ch = it->second;
            have = true;
        }
    }
    const char *env = std::getenv("CDNS_TUNE");
    if (!have && !force && env && std::strcmp(env, "0") == 0) {
        apply(c, Choice{});
        return CDNS_OK;
    }
    if (!have) {
        int r = measure(c, ch);
        if (r) return r;
        {
            std::lock_guard<std::mutex> lk(g_mu);
            g_wisdom[key] = ch;
        }
        if (wfile && *wfile && (r = cdns_wisdom_export(wfile))) return r;
    }
    apply(c, ch);
    return CDNS_OK;
}

}  // namespace cdns

using namespace cdns;

extern "C" {

int cdns_tune(cdns_ctx *c) {
    if (!c) return fail(CDNS_ERR_ARG, "null context");
    if (int r = require_whole(c)) return r;
    DeviceGuard guard(c->device);
    for (auto &g : c->graph)
        if (g) {
            cudaGraphExecDestroy(g);   // captured with the previous shapes
            g = nullptr;
        }
    int r = tune_context(c, true);
    if (r) return r;
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

int cdns_get_tuning(cdns_ctx *c, int *out) {
    if (!c || !out) return fail(CDNS_ERR_ARG, "null argument");
    out[0] = c->d.ztl;
    out[1] = c->t.yform & 1;
    out[2] = (c->t.yform >> 1) & 1;
    out[3] = c->d.xrw;
    return CDNS_OK;
}

int cdns_wisdom_export(const char *path) {
    if (!path) return fail(CDNS_ERR_ARG, "null path");
    std::ostringstream o;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        o << "{\"cdns_wisdom\": 1, \"entries\": [";
        bool first = true;
        for (const auto &kv : g_wisdom) {
            o << (first ? "" : ", ") << "{\"key\": \"" << kv.first << "\", \"ztl\": " << kv.second.ztl
              << ", \"yform\": " << kv.second.yform << ", \"xrw\": " << kv.second.xrw << "}";
            first = false;
        }
        o << "]}\n";
    }
    // write beside and rename, as the reference's wisdom export does
    const std::string tmp = std::string(path) + ".tmp";
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return fail(CDNS_ERR_ARG, std::string("cannot write ") + tmp);
        f << o.str();
        if (!f) return fail(CDNS_ERR_ARG, std::string("cannot write ") + tmp);
    }
    if (std::rename(tmp.c_str(), path) != 0) return fail(CDNS_ERR_ARG, std::string("cannot rename to ") + path);
    return CDNS_OK;
}

int cdns_wisdom_import(const char *path) {
    if (!path) return fail(CDNS_ERR_ARG, "null path");
    std::ifstream f(path);
    if (!f) return fail(CDNS_ERR_ARG, std::string("cannot read ") + path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string t = ss.str();
    if (t.find("\"cdns_wisdom\": 1") == std::string::npos) return fail(CDNS_ERR_ARG, "not a cdns wisdom file");
    std::map<std::string, Choice> got;
    size_t pos = 0;
    while ((pos = t.find("{\"key\": \"", pos)) != std::string::npos) {
        pos += 9;
        const size_t end = t.find('"', pos);
        if (end == std::string::npos) return fail(CDNS_ERR_ARG, "malformed wisdom entry");
        const std::string key = t.substr(pos, end - pos);
        Choice ch;
        int n = std::sscanf(t.c_str() + end, "\", \"ztl\": %d, \"yform\": %d, \"xrw\": %d}", &ch.ztl,
                            &ch.yform, &ch.xrw);
        if (n == 2) ch.xrw = 0;   // entries written before the x-stage choice existed
        if (n < 2 || ch.ztl < 0 || ch.ztl > 17 || (ch.ztl != 0 && ch.ztl < 8) || ch.yform < 0 || ch.yform > 3 ||
            (ch.xrw != 0 && (ch.xrw < 1 || ch.xrw > 5)))
            return fail(CDNS_ERR_ARG, "malformed wisdom entry");
        got[key] = ch;
        pos = end;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    for (const auto &kv : got) g_wisdom[kv.first] = kv.second;
    return CDNS_OK;
}

int cdns_wisdom_forget(void) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_wisdom.clear();
    return CDNS_OK;
}

}  // extern "C"
