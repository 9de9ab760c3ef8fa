"""Generate the golden fixtures in this folder from the reference's own sources.

Runs ``oracle/_ref/ref_runner`` (the reference C++ solver compiled from its
unmodified sources against the project FFTW/MPI shims; ``make -C oracle``)
on small seeded inputs and stores inputs and outputs as compressed npz files:

  golden_step.npz       16x17x16 channel (3/2 product grid), 4 steps from a
                        seeded divergence-free field: velocity and pressure.
  golden_example.npz    the reference's unit-test case shrunk to 16^3
                        (NXS=NZS=8, NYS=14, product grid = base grid, so the
                        Nyquist branches run; constant flow rate, wall
                        blowing 1e-3), 3 steps.
  golden_nonlinear.npz  nonlinear term N and pressure wall BC for a seeded
                        band-limited velocity (same shapes).
  golden_solve.npz      setup(g=150) + fused solve of a seeded RHS with
                        random wall data (NXS=5: a ragged x extent).
  golden_fine.npz       fine-grid backward/forward transforms of a band
                        spectrum on a 3/2 product grid.
  golden_coarse.npz     coarse-grid backward/forward transforms on a full
                        spectrum (Nyquist halve/mirror branches, 16x17x16)
                        and a ragged one (NXS=5, NZS=6): a realisable and an
                        arbitrary spectrum each.
  golden_files.npz      the reference's restart and physical files (field_S_,
                        field_P_; binary v1 and text) of a 16x17x16 state.
  golden_reduce.npz     the output branch on a 16x17x16 state (a divergence-free
                        field plus a non-solenoidal part): physical u, v, w,
                        p, plane sums, finite flags, EKT/TKE/div_L2.
  golden_blocks.npz     the reference Mesh's distributed block tables (x block,
                        fine-grid y slab, zero-mode owner) for 1..12 ranks on
                        four meshes, and the splits it rejects.
  golden_stats.npz      16x17x16 channel (log-law mean plus a k^-5/3
                        perturbation), 6 steps with Nstat = 2: the final
                        velocity and pressure and the Statistics running means
                        of the 4 sampled steps at full precision.

Usage: python tests/golden/make_golden.py [name ...]   (needs oracle/_ref built;
names: step example nonlinear solve fine coarse reduce files blocks stats, default all)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")]

import ref_io  # noqa: E402
from oracle_cases import band_spectrum, channel_case, divergence_free_field, example_case, orc  # noqa: E402


def mesh_dict(m, p):
    return dict(mesh=np.array([m.NX, m.NY, m.NZ, m.NXS, m.NYS, m.NZS, m.NX2, m.NY2, m.NZ2]),
                dom=np.array([m.XL, m.ZL]),
                parm=np.array([p.Re, p.G_pre, p.a_pre0, p.b_pre0, *p.a_V, *p.b_V,
                               p.INDEX_GRAD_PRE, p.THETA, p.DT, p.V_Microblow0]))


def coarse_and_reduce(which):
    if "coarse" in which:
        out = {}
        for tag, (m, p) in (("full", channel_case(16)),
                            ("ragged", example_case(NXS=5, NYS=14, NZS=6, N2=16, N=16))):
            rng = np.random.default_rng(51)
            realisable = orc.coarse_forward(m, rng.standard_normal((m.NZ, m.NY + 1, m.NX)))
            sh = m.spectral_shape()
            arbitrary = rng.standard_normal(sh) + 1j * rng.standard_normal(sh)
            for kind, U in (("real", realisable), ("arb", arbitrary)):
                phys, back = ref_io.coarse(m, p, U)
                out[f"{tag}_{kind}_U"], out[f"{tag}_{kind}_phys"], out[f"{tag}_{kind}_back"] = U, phys, back
            out[f"{tag}_mesh"] = mesh_dict(m, p)["mesh"]
            out[f"{tag}_dom"] = mesh_dict(m, p)["dom"]
            out[f"{tag}_parm"] = mesh_dict(m, p)["parm"]
        np.savez_compressed(os.path.join(HERE, "golden_coarse.npz"), **out)
    if "reduce" in which:
        m, p = channel_case(16)
        u = divergence_free_field(m, p, seed=61, amp=0.1, spectrum="k53", mean="loglaw")
        rng = np.random.default_rng(62)
        pres = orc.coarse_forward(m, rng.standard_normal((m.NZ, m.NY + 1, m.NX)))
        # a non-solenoidal part, so that the divergence norm is O(1) and not round-off
        u = [uc + orc.coarse_forward(m, 0.3 * rng.standard_normal((m.NZ, m.NY + 1, m.NX))) for uc in u]
        phys, planes, flags, values = ref_io.reduce(m, p, u, pres)
        np.savez_compressed(os.path.join(HERE, "golden_reduce.npz"), **mesh_dict(m, p), u=np.stack(u),
                            p=pres, phys=phys, planes=planes, flags=flags, values=values)


def dump_files(which):
    """golden_files.npz: the reference's restart and physical files (binary v1
    and text) of a 16x17x16 state, as byte arrays, with the state."""
    if "files" not in which:
        return
    m, p = channel_case(16)
    u = divergence_free_field(m, p, seed=71, amp=0.1, spectrum="k53", mean="loglaw")
    rng = np.random.default_rng(72)
    pres = orc.coarse_forward(m, rng.standard_normal((m.NZ, m.NY + 1, m.NX)))
    files = ref_io.dump(m, p, u, pres, 1234, 0.0625)
    np.savez_compressed(os.path.join(HERE, "golden_files.npz"), **mesh_dict(m, p), u=np.stack(u), p=pres,
                        ntpit=1234, time=0.0625,
                        **{k.replace(" ", "_").replace(".", "_"): np.frombuffer(v, dtype=np.uint8)
                           for k, v in files.items()})


BLOCK_CASES = {
    # tests/test_mesh.cpp:10-22 (32^3, NXS = NZS = 16, NYS = 30, 48^3 product grid)
    "distributed": lambda: example_case(NXS=16, NYS=30, NZS=16, N2=48, N=32),
    "channel32": lambda: channel_case(32),
    "retau180": lambda: channel_case(128),
    "narrow": lambda: example_case(NXS=1, NYS=6, NZS=2, N2=8, N=8),
}


def block_tables(which):
    if "blocks" not in which:
        return
    out = {}
    for tag, make in BLOCK_CASES.items():
        m, p = make()
        out[f"{tag}_mesh"] = mesh_dict(m, p)["mesh"]
        for ranks in range(1, 13):
            t = ref_io.blocks(m, p, ranks)
            out[f"{tag}_{ranks}"] = np.array([-1], dtype=np.int32) if t is None else t
    np.savez_compressed(os.path.join(HERE, "golden_blocks.npz"), **out)


def statistics_run(which):
    """golden_stats.npz: Simulation::run sampling Statistics at every step
    after Nstat (src/sim/simulation.cpp:225-250, src/sim/statistics.cpp:117-139)."""
    if "stats" not in which:
        return
    m, p = channel_case(16)
    u0 = divergence_free_field(m, p, seed=81, amp=0.1, spectrum="k53", mean="loglaw")
    ru, rp, _, st = ref_io.run_steps(m, p, u0, 6, nstat=2)
    np.savez_compressed(os.path.join(HERE, "golden_stats.npz"), **mesh_dict(m, p), nsteps=6, nstat=2,
                        u0=np.stack(u0), u=np.stack(ru), p=rp, count=st["count"],
                        dp_means=np.array(st["dp_means"]), means=st["means"])


def main(which):
    if not ref_io.available():
        raise SystemExit("oracle/_ref is not built: run make -C oracle")
    coarse_and_reduce(which)
    dump_files(which)
    block_tables(which)
    statistics_run(which)
    if "step" not in which:
        print("golden fixtures written to", HERE)
        return
    # 1. small channel, 4 steps
    m, p = channel_case(16)
    u0 = divergence_free_field(m, p, seed=11, amp=0.05, kmax=4)
    ru, rp, _ = ref_io.run_steps(m, p, u0, 4)
    np.savez_compressed(os.path.join(HERE, "golden_step.npz"), **mesh_dict(m, p), nsteps=4,
                        u0=np.stack(u0), u=np.stack(ru), p=rp)
    # 2. example case at 16^3 (full-spectrum Nyquist branch), 3 steps
    m, p = example_case(NXS=8, NYS=14, NZS=8, N2=16, N=16)
    u0 = [band_spectrum(m, s, 1e-3) for s in (21, 22, 23)]
    u0[0][m.NZS, :, 0] += np.array([1.5 * (v) for v in
                                    _cheb_1my2(m.ncy)])  # laminar mean 1.5(1-y^2)
    ru, rp, _ = ref_io.run_steps(m, p, u0, 3)
    np.savez_compressed(os.path.join(HERE, "golden_example.npz"), **mesh_dict(m, p), nsteps=3,
                        u0=np.stack(u0), u=np.stack(ru), p=rp)
    # 3. nonlinear term
    us = [band_spectrum(m, s, 0.1) for s in (4, 5, 6)]
    N, B = ref_io.nonlinear(m, p, us)
    np.savez_compressed(os.path.join(HERE, "golden_nonlinear.npz"), **mesh_dict(m, p),
                        u=np.stack(us), N=np.stack(N), B=np.stack(B))
    # 4. solve (Dirichlet walls; random wall data and RHS)
    m, p = example_case(NXS=5, NYS=14, NZS=8, N2=16, N=16)
    rng = np.random.default_rng(31)
    sh = m.spectral_shape()
    rv = [(rng.standard_normal(sh) + 1j * rng.standard_normal(sh)) * 1e-3 for _ in range(3)]
    bp = tuple((rng.standard_normal((m.nkz, m.nkx)) + 1j * rng.standard_normal((m.nkz, m.nkx))) * 1e-3
               for _ in range(2))
    bv = [tuple((rng.standard_normal((m.nkz, m.nkx)) + 1j * rng.standard_normal((m.nkz, m.nkx))) * 1e-3
                for _ in range(2)) for _ in range(3)]
    pres, vel, uu, wu = ref_io.solve(m, p, 150.0, rv, bp, bv)
    np.savez_compressed(os.path.join(HERE, "golden_solve.npz"), **mesh_dict(m, p), g=150.0,
                        rhs=np.stack(rv), bc_p=np.stack(bp), bc_v=np.array([np.stack(b) for b in bv]),
                        p=pres, v=np.stack(vel), u_unit=uu, w_unit=wu)
    # 5. fine transforms on a 3/2 grid
    m, p = channel_case(16)
    U = band_spectrum(m, 41)
    phys, back = ref_io.fine(m, p, U)
    np.savez_compressed(os.path.join(HERE, "golden_fine.npz"), **mesh_dict(m, p), U=U,
                        phys=phys, back=back)
    print("golden fixtures written to", HERE)


def _cheb_1my2(ncy):
    # 1 - y^2 = 0.5 T0 - 0.5 T2
    a = np.zeros(ncy)
    a[0] = 0.5
    a[2] = -0.5
    return a


if __name__ == "__main__":
    main(set(sys.argv[1:]) or {"step", "example", "nonlinear", "solve", "fine", "coarse", "reduce", "files",
                               "blocks", "stats"})
