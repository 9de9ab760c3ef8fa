// Restart and physical-field files in the reference's formats, written from
// and read into the device state (FieldIO::write_restart / read_restart /
// write_physical, src/io/field_io.cpp:121-427, single rank).
//
// Binary v1: a 128-byte little-endian header -- magic "CHDNS\0\0\0", u32
// version 1, u32 kind (1 restart, 2 physical), i64 step, f64 time, 12 i64
// dimensions (field_io.cpp:121-140) -- then the payload: the restart's
// velocity in the reference layout [kz][y][kx][3] as (re, im) doubles, the
// physical file's u, v, w, p planes [NZ][NY+1][NX].  Text: the first line
// "step time", then one "(re,im)" per restart value or one value per line
// (u v w per point, then p) for the physical file, every double in
// scientific notation with 17 digits.  The device produces the payload in the
// file's order (the interleave kernel, the coarse-grid snapshot), so the host
// only writes bytes; files are written beside and renamed, as the reference does.
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <string>
#include <vector>

#include "context.cuh"

namespace cdns {
namespace {

const unsigned char kMagic[8] = {'C', 'H', 'D', 'N', 'S', 0, 0, 0};
constexpr std::uint32_t kVersion = 1, kRestartKind = 1, kPhysicalKind = 2;
constexpr std::size_t kHeaderBytes = 128;

bool little_endian() {
    const std::uint32_t probe = 1;
    unsigned char b;
    std::memcpy(&b, &probe, 1);
    return b == 1;
}

void put_le(std::string &s, std::uint64_t v, int bytes) {
    for (int i = 0; i < bytes; ++i) s.push_back(static_cast<char>((v >> (8 * i)) & 0xff));
}

std::string header(std::uint32_t kind, long long step, double time, const long long (&dims)[12]) {
    std::string h(reinterpret_cast<const char *>(kMagic), 8);
    put_le(h, kVersion, 4);
    put_le(h, kind, 4);
    put_le(h, static_cast<std::uint64_t>(step), 8);
    std::uint64_t bits;
    std::memcpy(&bits, &time, 8);
    put_le(h, bits, 8);
    for (long long v : dims) put_le(h, static_cast<std::uint64_t>(v), 8);
    return h;
}

std::uint64_t get_le(const unsigned char *p, int bytes) {
    std::uint64_t v = 0;
    for (int i = 0; i < bytes; ++i) v |= static_cast<std::uint64_t>(p[i]) << (8 * i);
    return v;
}

// Write head + payload to path + ".tmp", then rename over path.
template <typename Fill> int atomic_write(const char *path, Fill fill) {
    const std::string tmp = std::string(path) + ".tmp";
    std::FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) return fail(CDNS_ERR_ARG, std::string("cannot open ") + tmp);
    const bool ok = fill(f);
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) {
        std::remove(tmp.c_str());
        return fail(CDNS_ERR_ARG, std::string("failed writing ") + tmp);
    }
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return fail(CDNS_ERR_ARG, std::string("cannot rename to ") + path);
    }
    return CDNS_OK;
}

// The velocity in the reference layout, on the host.
int velocity_host(cdns_ctx *c, std::vector<double> &v) {
    const size_t n = 3 * (size_t)c->d.Ns;
    v.resize(2 * n);
    launch_interleave(c->U[c->cur], c->aux, c->d.Ns, 3, c->stream);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(v.data(), c->aux, n * sizeof(double2), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return CDNS_OK;
}

// Parser of the reference's text restart (field_io.cpp:330-378): "step time"
// (an optional comma between), then "(re,im)" values, optional commas
// between them, Fortran exponents 'd'/'D' accepted.
struct TextReader {
    const std::string &t;
    size_t i = 0;
    void ws() {
        while (i < t.size() && std::isspace(static_cast<unsigned char>(t[i]))) ++i;
    }
    bool ch(char c) {
        ws();
        if (i < t.size() && t[i] == c) {
            ++i;
            return true;
        }
        return false;
    }
    bool number(double &v) {
        ws();
        std::string tok;
        while (i < t.size() && !std::isspace(static_cast<unsigned char>(t[i])) && t[i] != ')' && t[i] != ',')
            tok.push_back(t[i++]);
        for (char &x : tok)
            if (x == 'd' || x == 'D') x = 'e';
        if (tok.empty()) return false;
        char *end = nullptr;
        v = std::strtod(tok.c_str(), &end);
        return end == tok.c_str() + tok.size() && std::isfinite(v);
    }
    bool integer(long long &v) {
        ws();
        size_t j = i;
        while (j < t.size() && std::isdigit(static_cast<unsigned char>(t[j]))) ++j;
        if (j == i) return false;
        v = std::atoll(t.substr(i, j - i).c_str());
        i = j;
        return true;
    }
};

}  // namespace
}  // namespace cdns

using namespace cdns;

extern "C" {

int cdns_write_restart(cdns_ctx *c, const char *path, long long step, double time, int text) {
    if (!c || !path) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    if (!c->have_velocity) return fail(CDNS_ERR_STATE, "no velocity to write");
    if (!little_endian()) return fail(CDNS_ERR_ARG, "binary files need a little-endian host");
    DeviceGuard guard(c->device);
    std::vector<double> v;
    int r = velocity_host(c, v);
    if (r) return r;
    const Dims &d = c->d;
    const cdns_mesh_desc &m = c->mesh;
    if (text) {
        return atomic_write(path, [&](std::FILE *f) {
            bool ok = std::fprintf(f, "%lld %.17e\n", step, time) > 0;
            for (size_t k = 0; ok && k < v.size(); k += 2) ok = std::fprintf(f, "(%.17e,%.17e)\n", v[k], v[k + 1]) > 0;
            return ok;
        });
    }
    // field_io.cpp:125-140 with kind = restart, single rank (my_id 0, NPROC 1, x_begin 0)
    const long long dims[12] = {m.NX, m.NY + 1, m.NZ, 3, d.nkz, d.nkx, 0, 1, 0, d.nkx, 0, d.ncy};
    const std::string h = header(kRestartKind, step, time, dims);
    return atomic_write(path, [&](std::FILE *f) {
        return std::fwrite(h.data(), 1, h.size(), f) == h.size() &&
               std::fwrite(v.data(), sizeof(double), v.size(), f) == v.size();
    });
}

int cdns_read_restart(cdns_ctx *c, const char *path, long long *step, double *time) {
    if (!c || !path) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    std::ifstream in(path, std::ios::binary);
    if (!in) return fail(CDNS_ERR_ARG, std::string("cannot open restart: ") + path);
    std::string t((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    const Dims &d = c->d;
    const cdns_mesh_desc &m = c->mesh;
    const size_t nvals = 2 * 3 * (size_t)d.Ns;
    std::vector<double> v(nvals);
    long long s = 0;
    double tm = 0.0;
    if (t.size() >= 8 && std::memcmp(t.data(), kMagic, 8) == 0) {
        if (!little_endian()) return fail(CDNS_ERR_ARG, "binary files need a little-endian host");
        if (t.size() < kHeaderBytes) return fail(CDNS_ERR_ARG, "truncated field header");
        const unsigned char *p = reinterpret_cast<const unsigned char *>(t.data());
        if (get_le(p + 8, 4) != kVersion) return fail(CDNS_ERR_ARG, "unsupported field version");
        const std::uint32_t kind = (std::uint32_t)get_le(p + 12, 4);
        s = (long long)get_le(p + 16, 8);
        const std::uint64_t bits = get_le(p + 24, 8);
        std::memcpy(&tm, &bits, 8);
        const long long expect[12] = {m.NX, m.NY + 1, m.NZ, 3, d.nkz, d.nkx, 0, 1, 0, d.nkx, 0, d.ncy};
        bool dims_ok = true;
        for (int k = 0; k < 12; ++k) dims_ok = dims_ok && (long long)get_le(p + 32 + 8 * k, 8) == expect[k];
        if (kind != kRestartKind || s < 0 || !std::isfinite(tm) || !dims_ok)
            return fail(CDNS_ERR_ARG, "restart header does not match this rank and mesh");
        if (t.size() != kHeaderBytes + nvals * 8) return fail(CDNS_ERR_ARG, "restart payload length mismatch");
        std::memcpy(v.data(), t.data() + kHeaderBytes, nvals * 8);
        for (double x : v)
            if (!std::isfinite(x)) return fail(CDNS_ERR_ARG, "restart contains non-finite data");
    } else {
        TextReader rd{t};
        if (!rd.integer(s) || s < 0) return fail(CDNS_ERR_ARG, "invalid restart step");
        rd.ch(',');
        if (!rd.number(tm)) return fail(CDNS_ERR_ARG, "invalid text restart number");
        for (size_t k = 0; k < nvals; k += 2) {
            rd.ch(',');
            if (!rd.ch('(') || !rd.number(v[k]) || !rd.ch(',') || !rd.number(v[k + 1]) || !rd.ch(')'))
                return fail(CDNS_ERR_ARG, "invalid text complex syntax");
        }
        rd.ws();
        if (rd.i != t.size()) return fail(CDNS_ERR_ARG, "extra text restart data");
    }
    int r = cdns_set_velocity(c, v.data());
    if (r) return r;
    if (step) *step = s;
    if (time) *time = tm;
    return CDNS_OK;
}

int cdns_write_physical(cdns_ctx *c, const char *path, long long step, double time, int text) {
    if (!c || !path) return fail(CDNS_ERR_ARG, "null argument");
    if (int r = require_whole(c)) return r;
    if (!little_endian()) return fail(CDNS_ERR_ARG, "binary files need a little-endian host");
    const cdns_mesh_desc &m = c->mesh;
    const size_t plane = (size_t)m.NZ * (m.NY + 1) * m.NX;
    std::vector<double> phys(4 * plane);
    int r = cdns_output_reduce(c, 0, nullptr, nullptr, phys.data());
    if (r) return r;
    if (text) {
        // field_io.cpp:241-251: per point u v w (component fastest), then p
        return atomic_write(path, [&](std::FILE *f) {
            bool ok = std::fprintf(f, "%lld %.17e\n", step, time) > 0;
            for (size_t i = 0; ok && i < plane; ++i)
                ok = std::fprintf(f, "%.17e\n%.17e\n%.17e\n", phys[i], phys[plane + i], phys[2 * plane + i]) > 0;
            for (size_t i = 0; ok && i < plane; ++i) ok = std::fprintf(f, "%.17e\n", phys[3 * plane + i]) > 0;
            return ok;
        });
    }
    const long long dims[12] = {m.NX, m.NY + 1, m.NZ, 4, 0, 0, 0, 1, 0, m.NX, 0, m.NY + 1};
    const std::string h = header(kPhysicalKind, step, time, dims);
    return atomic_write(path, [&](std::FILE *f) {
        return std::fwrite(h.data(), 1, h.size(), f) == h.size() &&
               std::fwrite(phys.data(), sizeof(double), phys.size(), f) == phys.size();
    });
}

}  // extern "C"
