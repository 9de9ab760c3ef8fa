// Project-written driver around the reference's own, unmodified C++ sources
// (compiled from the reference tree with the FFTW/MPI shims in ref_shim/).
// Test infrastructure only: it produces golden vectors and the CPU baseline.
//
//   ref_runner run <run-dir> <out.bin> [threads] [stats.bin]
//       Params::load -> Mesh -> Transforms -> Simulation::initialize/run
//       (src/main.cpp:173-225 path), then writes nt, time, the spectral
//       velocity [kz][y][kx][3] and pressure [kz][y][kx] (complex<double>).
//       Prints the step-loop wall time (steady_clock, as src/main.cpp:224-233).
//       With stats.bin, also writes the run's Statistics running means at
//       full precision (the values Statistics::write prints with 8 decimals,
//       src/sim/statistics.cpp:117-139, :163-205): int64 count, dpdx mean,
//       dpdz mean, then per y plane-array of NY+1 doubles in the order
//       u v w, p, uu vv ww uv vw wu, pp, pu pv pw, u^3 v^3 w^3, u^4 v^4 w^4.
//   ref_runner nonlinear <run-dir> <velocity.bin> <out.bin>
//       TimeStepper::nonlinear_term (src/solver/timestepper.cpp:11-17):
//       writes N [kz][y][kx][3] and the pressure wall BC [kz][2][kx].
//   ref_runner fine <run-dir> <spectral.bin> <out.bin>
//       Transforms::channel_xyzfft2 'B' then 'F' of one scalar field
//       (src/fft/transforms.cpp:615-741): writes physical then spectral.
//   ref_runner coarse <run-dir> <spectral.bin> <out.bin>
//       Transforms::channel_xyzfft 'B' then 'F' of one scalar field
//       (src/fft/transforms.cpp:452-582): writes physical then spectral.
//   ref_runner reduce <run-dir> <state.bin> <out.bin>
//       The output branch of Simulation::run (src/sim/simulation.cpp:226-235)
//       on a given velocity [kz][y][kx][3] and pressure [kz][y][kx]:
//       FieldIO::to_physical, Statistics::reduce(higher, validate) and
//       Diagnostics::evaluate; writes the physical u, v, w, p, the plane sums
//       [NY+1][20], the plane finite flags and (EKT, TKE, div_L2, finite).
//   ref_runner dump <run-dir> <state.bin> <ntpit> <time>
//       FieldIO (format "both") on a given velocity and pressure: write_restart
//       and, of the to_physical snapshot, write_physical, into <run-dir>
//       (src/io/field_io.cpp:241-309): field_S_ 0.bin/.dat, field_P_ 0.bin/.dat.
//   ref_runner solve <run-dir> <g> <rhs.bin> <out.bin>
//       EqSolvePV::setup(g) then the fused solve_modes with fused RHS and
//       sigma correction (src/solver/eqsolve_pv.cpp:311-450); input is the
//       velocity RHS [kz][y][kx][3], pressure BC [kz][2][kx], velocity BC
//       [kz][2][kx][3]; writes pressure, velocity, u_dpdx_unit, w_dpdz_unit.
//   ref_runner blocks <run-dir> <ranks> <out.bin>
//       The distributed block tables of Mesh (src/core/mesh.cpp:20-85) for a
//       <ranks>-way split (INDEX_Serial = 0): per rank, int32 x_begin,
//       x_count, y2_begin, y2_count, owns_zero_x_mode; or a single int32 -1
//       if Mesh rejects the split.
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "core/cpu_device.hpp"
#include "core/mesh.hpp"
#include "core/mpi_context.hpp"
#include "core/params.hpp"
#include "fft/transforms.hpp"
#include "io/field_io.hpp"
#include "sim/diagnostics.hpp"
#include "sim/simulation.hpp"
#include "sim/statistics.hpp"
#include "solver/eqsolve_pv.hpp"
#include "solver/fields.hpp"
#include "solver/timestepper.hpp"

// Friend hook declared by the reference (src/solver/eqsolve_pv.hpp:11,34).
struct EqSolvePVTestAccess {
    static void solve(EqSolvePV &s, ScalarField &p, const ScalarBoundary &pbc, VectorField &v,
                      const VectorField &rhs, const VectorBoundary &vbc) {
        s.solve_modes(p, nullptr, pbc, v, rhs, vbc, true);
    }
};

// Read access to the running means that Simulation keeps in its Statistics
// member (src/sim/simulation.hpp:66, src/sim/statistics.hpp:34-40), which the
// reference only prints rounded to 8 decimals.  Names used in an explicit
// instantiation are exempt from access checking ([temp.explicit]), so each
// Member<Tag, &Class::member_> instantiation defines a friend get(Tag) that
// returns the member pointer.
namespace member_access {
template <typename Tag, typename Tag::type Ptr> struct Member {
    friend typename Tag::type get(Tag) { return Ptr; }
};
struct SimStatistics { using type = Statistics Simulation::*; friend type get(SimStatistics); };
struct StatsVector { using type = std::vector<double> Statistics::*; };
struct VelocityMean : StatsVector { friend type get(VelocityMean); };
struct PressureMean : StatsVector { friend type get(PressureMean); };
struct VelocitySecond : StatsVector { friend type get(VelocitySecond); };
struct PressureVelocity : StatsVector { friend type get(PressureVelocity); };
struct PressureSecond : StatsVector { friend type get(PressureSecond); };
struct VelocityThird : StatsVector { friend type get(VelocityThird); };
struct VelocityFourth : StatsVector { friend type get(VelocityFourth); };
template struct Member<SimStatistics, &Simulation::statistics_>;
template struct Member<VelocityMean, &Statistics::velocity_mean_>;
template struct Member<PressureMean, &Statistics::pressure_mean_>;
template struct Member<VelocitySecond, &Statistics::velocity_second_>;
template struct Member<PressureVelocity, &Statistics::pressure_velocity_>;
template struct Member<PressureSecond, &Statistics::pressure_second_>;
template struct Member<VelocityThird, &Statistics::velocity_third_>;
template struct Member<VelocityFourth, &Statistics::velocity_fourth_>;
}  // namespace member_access

namespace {
template <typename T> void read_all(const std::string &path, std::vector<T> &out) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("cannot open " + path);
    in.seekg(0, std::ios::end);
    const auto bytes = static_cast<std::size_t>(in.tellg());
    in.seekg(0);
    if (bytes != out.size() * sizeof(T))
        throw std::runtime_error(path + ": expected " + std::to_string(out.size() * sizeof(T)) +
                                 " bytes, found " + std::to_string(bytes));
    in.read(reinterpret_cast<char *>(out.data()), static_cast<std::streamsize>(bytes));
}

template <typename T> void write(std::ofstream &out, const T *data, std::size_t n) {
    out.write(reinterpret_cast<const char *>(data), static_cast<std::streamsize>(n * sizeof(T)));
}

void fill(Array4D<std::complex<double>> &f, const std::complex<double> *src) {
    std::copy(src, src + f.size(), f.data());
}
}  // namespace

int main(int argc, char **argv) {
    if (argc < 4) {
        std::cerr << "usage: ref_runner run|nonlinear|fine|coarse|reduce|dump|solve|blocks <run-dir> ...\n";
        return 2;
    }
    const std::string mode = argv[1];
    const std::string dir = argv[2];
    try {
        int threads = 1;
        if (mode == "run" && argc > 4) threads = std::atoi(argv[4]);
        cpu_device(threads);
        MpiContext mpi(MPI_COMM_WORLD);
        Params params = Params::load(dir);
        Mesh mesh(params.mesh, params.parm.XL, params.parm.ZL, 0, 1);
        Transforms fft(mesh, params.parm.XL, params.parm.ZL, params.parm.Re, "", &mpi);
        if (mode == "run") {
            Simulation sim(params, mesh, fft, dir, &mpi);
            sim.initialize();
            const auto start = std::chrono::steady_clock::now();
            sim.run();
            const double wall =
                std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count();
            std::cout << "ref_runner: steps " << params.ctrl.NSTEPS << " wall " << wall
                      << " s threads " << threads << "\n";
            std::ofstream out(argv[3], std::ios::binary);
            const std::int64_t nt = sim.nt();
            const double t = sim.time();
            write(out, &nt, 1);
            write(out, &t, 1);
            write(out, sim.velocity().data(), sim.velocity().size());
            write(out, sim.pressure().data(), sim.pressure().size());
            if (argc > 5) {
                namespace ma = member_access;
                const Statistics &st = sim.*get(ma::SimStatistics{});
                std::ofstream so(argv[5], std::ios::binary);
                const std::int64_t count = st.count();
                const double dp[2] = {st.dpdx_mean(), st.dpdz_mean()};
                write(so, &count, 1);
                write(so, dp, 2);
                for (const auto &v : {st.*get(ma::VelocityMean{}), st.*get(ma::PressureMean{}),
                                      st.*get(ma::VelocitySecond{}), st.*get(ma::PressureSecond{}),
                                      st.*get(ma::PressureVelocity{}), st.*get(ma::VelocityThird{}),
                                      st.*get(ma::VelocityFourth{})})
                    write(so, v.data(), v.size());
                if (!so) return 1;
            }
            return out ? 0 : 1;
        }
        if (mode == "nonlinear" && argc >= 5) {
            EqSolvePV solver(params, mesh, fft);
            TimeStepper stepper(params, mesh, fft, solver);
            VectorField velocity = make_vector_field(mesh), nl = make_vector_field(mesh);
            ScalarBoundary bc = make_scalar_boundary(mesh);
            std::vector<std::complex<double>> buf(velocity.size());
            read_all(argv[3], buf);
            fill(velocity, buf.data());
            stepper.nonlinear_term(nl, velocity, bc);
            std::ofstream out(argv[4], std::ios::binary);
            write(out, nl.data(), nl.size());
            write(out, bc.data(), bc.size());
            return out ? 0 : 1;
        }
        if (mode == "fine" && argc >= 5) {
            ScalarField spec = make_scalar_field(mesh), back = make_scalar_field(mesh);
            std::vector<std::complex<double>> buf(spec.size());
            read_all(argv[3], buf);
            fill(spec, buf.data());
            std::vector<double> phys(static_cast<std::size_t>(mesh.NZ2) * (mesh.NY2P + 1) *
                                     mesh.NX2);
            fft.channel_xyzfft2('B', phys.data(), spec.data());
            fft.channel_xyzfft2('F', phys.data(), back.data());
            std::ofstream out(argv[4], std::ios::binary);
            write(out, phys.data(), phys.size());
            write(out, back.data(), back.size());
            return out ? 0 : 1;
        }
        if (mode == "coarse" && argc >= 5) {
            ScalarField spec = make_scalar_field(mesh), back = make_scalar_field(mesh);
            std::vector<std::complex<double>> buf(spec.size());
            read_all(argv[3], buf);
            fill(spec, buf.data());
            std::vector<double> phys(static_cast<std::size_t>(mesh.NZ) * (mesh.NYP + 1) * mesh.NX);
            fft.channel_xyzfft('B', phys.data(), spec.data());
            fft.channel_xyzfft('F', phys.data(), back.data());
            std::ofstream out(argv[4], std::ios::binary);
            write(out, phys.data(), phys.size());
            write(out, back.data(), back.size());
            return out ? 0 : 1;
        }
        if (mode == "reduce" && argc >= 5) {
            VectorField velocity = make_vector_field(mesh);
            ScalarField pressure = make_scalar_field(mesh);
            std::vector<std::complex<double>> buf(velocity.size() + pressure.size());
            read_all(argv[3], buf);
            fill(velocity, buf.data());
            fill(pressure, buf.data() + velocity.size());
            FieldIO io(mesh, fft, dir, &mpi);
            bool finite = true;
            const auto &snapshot = io.to_physical(velocity, pressure, &finite);
            Statistics stats(mesh);
            const auto &planes = stats.reduce(snapshot.velocity, snapshot.pressure, true, true);
            Diagnostics diag(mesh, fft, &mpi);
            const auto values = diag.evaluate(planes, velocity, finite);
            std::ofstream out(argv[4], std::ios::binary);
            for (int c = 0; c < 3; ++c) write(out, snapshot.velocity[c].data(), snapshot.velocity[c].size());
            write(out, snapshot.pressure.data(), snapshot.pressure.size());
            for (const auto &pl : planes) write(out, pl.sum.data(), pl.sum.size());
            for (const auto &pl : planes) {
                const double f = pl.finite ? 1.0 : 0.0;
                write(out, &f, 1);
            }
            const double v[4] = {values.ekt, values.tke, values.divergence_l2, values.finite ? 1.0 : 0.0};
            write(out, v, 4);
            return out ? 0 : 1;
        }
        if (mode == "dump" && argc >= 6) {
            VectorField velocity = make_vector_field(mesh);
            ScalarField pressure = make_scalar_field(mesh);
            std::vector<std::complex<double>> buf(velocity.size() + pressure.size());
            read_all(argv[3], buf);
            fill(velocity, buf.data());
            fill(pressure, buf.data() + velocity.size());
            const std::int64_t ntpit = std::atoll(argv[4]);
            const double t = std::atof(argv[5]);
            FieldIO io(mesh, fft, dir, &mpi, OutputFormat::Both);
            const auto &snapshot = io.to_physical(velocity, pressure, nullptr);
            io.write_restart(ntpit, t, velocity);
            io.write_physical(ntpit, t, snapshot);
            return 0;
        }
        if (mode == "blocks" && argc >= 5) {
            const int ranks = std::atoi(argv[3]);
            MeshParm mp = params.mesh;
            mp.INDEX_Serial = 0;
            std::vector<std::int32_t> table;
            try {
                for (int r = 0; r < ranks; ++r) {
                    Mesh m(mp, params.parm.XL, params.parm.ZL, r, ranks);
                    table.insert(table.end(), {m.x_begin(r), m.x_count(r), m.y2_begin(r), m.y2_count(r),
                                               m.owns_zero_x_mode() ? 1 : 0});
                }
            } catch (const std::invalid_argument &) {
                table.assign(1, -1);
            }
            std::ofstream out(argv[4], std::ios::binary);
            write(out, table.data(), table.size());
            return out ? 0 : 1;
        }
        if (mode == "solve" && argc >= 6) {
            const double g = std::atof(argv[3]);
            EqSolvePV solver(params, mesh, fft);
            solver.setup(g);
            VectorField rhs = make_vector_field(mesh), vel = make_vector_field(mesh);
            ScalarField pres = make_scalar_field(mesh);
            ScalarBoundary pbc = make_scalar_boundary(mesh);
            VectorBoundary vbc = make_vector_boundary(mesh);
            std::vector<std::complex<double>> buf(rhs.size() + pbc.size() + vbc.size());
            read_all(argv[4], buf);
            fill(rhs, buf.data());
            fill(pbc, buf.data() + rhs.size());
            fill(vbc, buf.data() + rhs.size() + pbc.size());
            EqSolvePVTestAccess::solve(solver, pres, pbc, vel, rhs, vbc);
            std::ofstream out(argv[5], std::ios::binary);
            write(out, pres.data(), pres.size());
            write(out, vel.data(), vel.size());
            write(out, solver.u_dpdx_unit().data(), solver.u_dpdx_unit().size());
            write(out, solver.w_dpdz_unit().data(), solver.w_dpdz_unit().size());
            return out ? 0 : 1;
        }
        std::cerr << "ref_runner: bad arguments\n";
        return 2;
    } catch (const std::exception &e) {
        std::cerr << "ref_runner: " << e.what() << "\n";
        return 1;
    }
}
