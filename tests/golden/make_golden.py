"""Generate the golden fixtures of tests/golden/ by running the reference's own C++.

The reference (NNPEngine src/, compiled in place by oracle/Makefile into oracle/_ref/ref_dump)
is run on the seeded cases of tests/cases.py; its outputs are stored compactly:

* water648.npz   648-atom water box (6^3 molecules, 18.624 A): per-atom full-list counts and
                 digests of the sorted (id_j, image, special) keys; forces and energy/virial of one
                 force evaluation (pair + bond + angle); cell-based and list-based g(r) counts; a
                 20-step NVE trajectory in the reference's float arithmetic (final x, v and the
                 per-step energies).
* nnp_gauss648.npz  the same box under the reference's tabulated NNP (NNPOTENTIAL_TBL, 6 A, 750
                 bins, 20 Gaussians per pair type and special class, pair part from coef_p) with a
                 20->32->32->1 fitting network evaluated by the TF C-API shim: descriptor, dE/dG,
                 network energy, forces (bonded + NNP).
* mixture2000.npz  2000-atom two-species LJ+Coulomb liquid at 0.035 A^-3: g(r) counts to 15 A in
                 0.01 A bins, the reference's float g(r) and S(q) on 512 q points, forces.
* rmdf2000.npz   the same liquid with RMDF (grsq.cpp:899-1377) against a seeded synthetic S(q)
                 target (strength 0.02, gamma 0.5): the refined force/potential tables, weighted
                 S(q) and penalty of one update on the snapshot's S(q); and a 20-step NVE run with
                 g(r) steps every 5 steps (cell-based every 10): per-log-step penalty, final x, v
                 and tables.

* driver648.npz  the reference's own executable (oracle/_ref/nnp.exe: run.cpp + main.cpp, unmodified)
                 on run input files of both modes for the 648-atom water box at 0 K (so that the
                 first log line does not depend on its unseeded generator): the classical mode with
                 RMDF (strength 0.02, gamma 0.5) and the nnp_run mode with the tabulated NNP and RMDF
                 on its pair tables; its log lines and the line counts of its output files.

* sqd648.npz, sqd2000.npz  the reference's direct S(q) (SQD, grsq.cpp:362-585) of the 648-atom water
                 box (jittered, 60 bins to 6 A^-1) and of the 2000-atom mixture (40 bins to 3 A^-1):
                 the positions it used, mean |G| per bin, S(q) per type pair and G count per bin.

Run:  python tests/golden/make_golden.py [name ...]   (needs the reference's sources, found by
oracle.orc.refsrc(), and the harness that oracle.orc.build() compiles from them; without names
every fixture is written).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

from oracle import orc  # noqa: E402
import cases  # noqa: E402


def bonded_cfg():
    return {"bond": [f"1.0 {cases.WATER_BOND_K}"], "angle": [f"109.47 0 0 {cases.WATER_ANGLE_KC}"]}


def water648(work):
    s, table = cases.water_case()
    f = cases.write_inputs(s, table, work)
    v0 = os.path.join(work, "v0.bin")
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    base = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10, **bonded_cfg()}
    snap = orc.run_ref_dump({**base, "velocity": v0, "mode": "snapshot"}, os.path.join(work, "snap"))
    counts, digests = cases.list_keys(snap["fulllist"], s.natom)
    md = orc.run_ref_dump({**base, "velocity": f["vel"], "mode": "md", "steps": 20, "dt": 1, "log_interval": 1},
                          os.path.join(work, "md"))
    out = dict(x=s.x, v=s.v, list_counts=counts, list_digests=digests, nghost=snap["info"]["nghost"],
               force=snap["force"].reshape(-1, 3), erg_f32=snap["log_e"], vir_f32=snap["log_w"],
               gr_counts=snap["gr_counts"].reshape(3, -1), gr_inner_counts=snap["gr_inner_counts"].reshape(3, -1),
               md_x=md["x"].reshape(-1, 3), md_v=md["v"].reshape(-1, 3), md_erg=md["log_e"], md_ekin=md["log_k"],
               md_nbuild=md["info"]["nbuild_last"])
    np.savez_compressed(os.path.join(HERE, "water648.npz"), **out)
    print("water648:", s.natom, "atoms,", int(counts.sum()), "list entries,", snap["info"]["nghost"], "images")


def mixture2000(work):
    s, table = cases.mixture_case()
    f = cases.write_inputs(s, table, work)
    v0 = os.path.join(work, "v0.bin")
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    snap = orc.run_ref_dump({"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2,
                             "gr_cutoff": 15, "nq": 512, "qmax": 20, "velocity": v0, "mode": "snapshot"},
                            os.path.join(work, "snap"))
    counts, digests = cases.list_keys(snap["fulllist"], s.natom)
    out = dict(x=s.x, v=s.v, typ=s.typ, list_counts=counts, list_digests=digests,
               force=snap["force"].reshape(-1, 3), erg_f32=snap["log_e"],
               gr_counts=snap["gr_counts"].reshape(3, -1), gr_inner_counts=snap["gr_inner_counts"].reshape(3, -1),
               gr_f32=snap["gr"].reshape(3, -1), sq_f32=snap["sq"].reshape(3, -1), qq=snap["qq"])
    np.savez_compressed(os.path.join(HERE, "mixture2000.npz"), **out)
    print("mixture2000:", s.natom, "atoms, gr bins", out["gr_counts"].shape)


RMDF_STRENGTH, RMDF_GAMMA = 0.02, 0.5


def rmdf_target(work, ntype=2):
    from nnpengine_b200 import systems as S
    q, sqex, wt, ff = S.synthetic_sq_target(512, 20.0, ntype, seed=7)
    path = os.path.join(work, "sq_target.txt")
    S.write_sq_target(path, q, sqex, wt, ff)
    return path, (q, sqex, wt, ff)


def rmdf2000(work):
    s, table = cases.mixture_case()
    f = cases.write_inputs(s, table, work)
    v0 = os.path.join(work, "v0.bin")
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    tpath, (q, sqex, wt, ff) = rmdf_target(work)
    base = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 15, "nq": 512,
            "qmax": 20, "rmdf": f"{RMDF_STRENGTH} {RMDF_GAMMA} {tpath}"}
    snap = orc.run_ref_dump({**base, "velocity": v0, "mode": "snapshot"}, os.path.join(work, "snap"))
    md = orc.run_ref_dump({**base, "velocity": f["vel"], "mode": "md", "steps": 20, "dt": 1, "log_interval": 5,
                           "gr_interval": "5 10"}, os.path.join(work, "md"))
    out = dict(sqex=sqex, wt=wt, ff=ff, q=q, tbl_force=snap["tbl_force"].reshape(3, -1), tbl_pot=snap["tbl_pot"].reshape(3, -1),
               rmdf_sq=snap["rmdf_sq"], rmdf_erg=snap["rmdf_erg"], sq_f32=snap["sq"].reshape(3, -1),
               md_x=md["x"].reshape(-1, 3), md_v=md["v"].reshape(-1, 3), md_erg=md["log_e"], md_exp=md["log_exp"],
               md_tbl_force=md["tbl_force"].reshape(3, -1), md_tbl_pot=md["tbl_pot"].reshape(3, -1))
    np.savez_compressed(os.path.join(HERE, "rmdf2000.npz"), **out)
    print("rmdf2000: penalty", float(snap["rmdf_erg"][0]), "md penalties", md["log_exp"])


def driver648(work):
    import subprocess
    from nnpengine_b200 import nnp_model as NM
    out = {}
    for mode in ("classical", "nnp_run"):
        d = os.path.join(work, mode)
        os.makedirs(d, exist_ok=True)
        s, table = cases.water_case()
        tpath, _ = rmdf_target(d)
        if mode == "classical":
            path, files = cases.write_run_input(d, mode, s, table, rmdf=(RMDF_STRENGTH, RMDF_GAMMA, tpath))
        else:
            paths = cases.write_nnp_inputs(NM.gauss_model(), d)
            path, files = cases.write_run_input(d, mode, s, nnp_paths=paths, rmdf=(RMDF_STRENGTH, RMDF_GAMMA, tpath),
                                                nbin=750, cutoffs=(6.0, 2.0, 6.0))
        r = subprocess.run([os.path.join(orc.REF_DIR, "nnp.exe"), mode, path], capture_output=True, text=True,
                           timeout=600, check=True)
        out[f"{mode}_log"] = cases.parse_log(r.stdout)
        out[f"{mode}_lines"] = np.array([sum(1 for _ in open(files[k])) if os.path.exists(files[k]) else 0
                                         for k in ("xyz", "gr", "sq", "sqx", "force")])
        print(f"driver648 {mode}: step 0 {out[f'{mode}_log'][0]}, output lines {out[f'{mode}_lines']}")
    np.savez_compressed(os.path.join(HERE, "driver648.npz"), **out)


def nnp_gauss648(work):
    from nnpengine_b200 import nnp_model as NM
    s, table = cases.water_case()
    f = cases.write_inputs(s, table, work)
    v0 = os.path.join(work, "v0.bin")
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    m = NM.gauss_model()
    paths = cases.write_nnp_inputs(m, work)
    snap = orc.run_ref_dump({"init": f["init"], "no_lj": "", "nnp": f"6.0 750 {paths['param']} {paths['wt']}",
                             "skin": 2, "gr_cutoff": 6, "bond": ["1.0 0"], "angle": ["109.47 0 0 0"],
                             "velocity": v0, "mode": "snapshot"}, os.path.join(work, "snap"))
    out = dict(x=s.x, desc=snap["desc"].reshape(s.natom, 20), dedg=snap["dedg"].reshape(s.natom, 20),
               force=snap["force"].reshape(-1, 3), f_bonded=snap["f_classical"].reshape(-1, 3),
               erg_f32=snap["log_e"], enn=snap["log_enn"])
    np.savez_compressed(os.path.join(HERE, "nnp_gauss648.npz"), **out)
    print("nnp_gauss648: network energy", float(snap["log_enn"][0]))


def _sqd_fixture(work, name, s, table, nq, qmax):
    f = cases.write_inputs(s, table, work)
    cfg = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10,
           "velocity": f["vel"], "mode": "md", "steps": 0, "dt": 0.5, "log_interval": 1, "sqd": f"{nq} {qmax}"}
    if s.moltypes[0].n_atom > 1:
        cfg.update(bonded_cfg())
    r = orc.run_ref_dump(cfg, work)
    out = dict(x=r["x"].reshape(-1, 3), typ=s.typ, bl=np.float32(s.bl), nq=nq, qmax=np.float32(qmax),
               q=r["sqd_q"], sq=r["sqd_sq"].reshape(nq, -1), count=r["sqd_count"], ngv=r["info"]["sqd_ngv"])
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
    print(name + ":", s.natom, "atoms,", out["ngv"], "G vectors")


def sqd648(work):
    s, table = cases.water_case(jitter=0.05)
    _sqd_fixture(work, "sqd648", s, table, 60, 6.0)


def sqd2000(work):
    s, table = cases.mixture_case()
    _sqd_fixture(work, "sqd2000", s, table, 40, 3.0)


def water3000(work):
    """The 3000-atom water box of the plain workload (1000 molecules on a 10^3 lattice, 31.04 A box,
    seed 2, 300 K Maxwell-Boltzmann): the reference's snapshot (list, images, forces, energies, g(r)
    counts), 100 and 1000 NVE steps at 1 fs (energies every 10 steps, final x and v), and 5 ps at
    1 fs under its Andersen thermostat at 300 K (the equilibrated state the network workload starts
    from)."""
    s, table = cases.water3000_case()
    f = cases.write_inputs(s, table, work)
    base = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10,
            "velocity": f["vel"], **bonded_cfg()}
    v0 = os.path.join(work, "v0.bin")     # the snapshot at rest: its positions are the input's exactly
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    snap = orc.run_ref_dump({**base, "velocity": v0, "mode": "snapshot"}, os.path.join(work, "snap"))
    counts, digests = cases.list_keys(snap["fulllist"], s.natom)
    md = {"mode": "md", "dt": 1, "log_interval": 10}
    m100 = orc.run_ref_dump({**base, **md, "steps": 100}, os.path.join(work, "m100"))
    m1000 = orc.run_ref_dump({**base, **md, "steps": 1000}, os.path.join(work, "m1000"))
    eq = orc.run_ref_dump({**base, "mode": "md", "dt": 1, "log_interval": 1000, "steps": 5000, "temp": 300,
                           "scale_interval": 10, "seed": 31}, os.path.join(work, "eq"))
    out = dict(x=s.x, v=s.v, list_counts=counts, list_digests=digests, nghost=snap["info"]["nghost"],
               force=snap["force"].reshape(-1, 3), erg_f32=snap["log_e"], vir_f32=snap["log_w"],
               gr_counts=snap["gr_counts"].reshape(3, -1), gr_inner_counts=snap["gr_inner_counts"].reshape(3, -1),
               md100_x=m100["x"].reshape(-1, 3), md100_v=m100["v"].reshape(-1, 3), md100_erg=m100["log_e"],
               md100_ekin=m100["log_k"], md100_nbuild=m100["info"]["nbuild_last"],
               md1000_erg=m1000["log_e"], md1000_ekin=m1000["log_k"], md1000_nbuild=m1000["info"]["nbuild_last"],
               eq_x=eq["x"].reshape(-1, 3), eq_v=eq["v"].reshape(-1, 3), eq_ekin=eq["log_k"])
    np.savez_compressed(os.path.join(HERE, "water3000.npz"), **out)
    print("water3000:", s.natom, "atoms,", int(counts.sum()), "list entries,", snap["info"]["nghost"], "images;",
          "1000-step nbuild", m1000["info"]["nbuild_last"], "; equilibrated T",
          float(eq["log_k"][-1]) / s.natom * 2 / 3 / 0.0019872)


def mixture30k(work):
    """The 30,000-atom two-species liquid of the g(r)/S(q) workload (0.035 A^-3, seed 4): the
    reference's g(r) counts to 15 A (cell-based) and to the list cutoff (list-based), its float
    S(q), the list counts with block digests, the image count; and the RMDF target: the weighted
    S(q) (RMDF's sq, what RMDF::dumpSQ writes) of the same liquid with every eps x1.1 after 500
    steps at 1 fs under its Andersen thermostat at 300 K (seed 41)."""
    from nnpengine_b200 import systems as S
    s, table = cases.mixture30k_case()
    f = cases.write_inputs(s, table, work)
    v0 = os.path.join(work, "v0.bin")
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    snap = orc.run_ref_dump({"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2,
                             "gr_cutoff": 15, "nq": 512, "qmax": 20, "velocity": v0, "mode": "snapshot"},
                            os.path.join(work, "snap"))
    counts, digests = cases.list_keys(snap["fulllist"], s.natom)
    # target: eps x1.1 table, g(r) step (cell-based) at md_step 0 and 500, RMDF of strength 0
    r, F11, U11 = cases.mixture_table(eps_scale=1.1)
    t11 = os.path.join(work, "table11.txt")
    S.write_pair_table(t11, r, F11, U11)
    q, sqex, wt, ff = S.synthetic_sq_target(512, 20.0, 2)
    tpath = os.path.join(work, "sq_dummy.txt")
    S.write_sq_target(tpath, q, sqex, wt, ff)
    tgt = orc.run_ref_dump({"init": f["init"], "table": f"1000 {t11}", "cutoff": 10, "skin": 2, "gr_cutoff": 15,
                            "nq": 512, "qmax": 20, "velocity": f["vel"], "mode": "md", "dt": 1, "steps": 500,
                            "log_interval": 500, "temp": 300, "scale_interval": 10, "seed": 41,
                            "gr_interval": "500 500", "rmdf": f"0 1 {tpath}"}, os.path.join(work, "tgt"))
    out = dict(x_digest=cases.x_digest(s.x), natom=s.natom, list_counts=counts.astype(np.int32),
               list_block_digests=cases.block_digests(digests), nghost=snap["info"]["nghost"],
               gr_counts=snap["gr_counts"].reshape(3, -1), gr_inner_counts=snap["gr_inner_counts"].reshape(3, -1),
               sq_f32=snap["sq"].reshape(3, -1), erg_f32=snap["log_e"],
               target_sq=tgt["rmdf_sq"].astype(np.float32), target_q=q, target_wt=wt, target_ff=ff)
    np.savez_compressed(os.path.join(HERE, "mixture30k.npz"), **out)
    print("mixture30k:", s.natom, "atoms,", int(counts.sum()), "list entries; ordered pairs in the 15 A tally",
          int(out["gr_counts"].sum()))


def peroxide2048(work):
    """512 H2O2 molecules (2048 atoms, 30.4 A box, seed 9, jittered 0.05 A) with bonds, angles and
    the H-O-O-H dihedral: the reference's forces and energies with the water pair table, and its
    bonded terms alone (no pair term), plus 20 NVE steps at 0.5 fs."""
    s, table = cases.peroxide_case()
    f = cases.write_inputs(s, table, work)
    bcfg = cases.peroxide_bonded_cfg()
    v0 = os.path.join(work, "v0.bin")
    np.zeros((s.natom, 3), np.float32).tofile(v0)
    base = {"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2, "gr_cutoff": 10, **bcfg}
    snap = orc.run_ref_dump({**base, "velocity": v0, "mode": "snapshot"}, os.path.join(work, "snap"))
    bond = orc.run_ref_dump({**base, "no_lj": "", "velocity": v0, "mode": "snapshot"}, os.path.join(work, "bond"))
    md = orc.run_ref_dump({**base, "velocity": f["vel"], "mode": "md", "steps": 20, "dt": 0.5, "log_interval": 1},
                          os.path.join(work, "md"))
    out = dict(x=s.x, v=s.v, force=snap["force"].reshape(-1, 3), erg_f32=snap["log_e"],
               f_bonded=bond["force"].reshape(-1, 3), erg_bonded=bond["log_e"],
               md_x=md["x"].reshape(-1, 3), md_v=md["v"].reshape(-1, 3), md_erg=md["log_e"], md_ekin=md["log_k"])
    np.savez_compressed(os.path.join(HERE, "peroxide2048.npz"), **out)
    print("peroxide2048: bonded energy", float(bond["log_e"][0]), "total", float(snap["log_e"][0]))


def dumps648(work):
    """Content of the reference executable's output files (oracle/_ref/nnp.exe, run.cpp + main.cpp
    unmodified) in both modes for the 648-atom water box: total_steps 0 at 0 K, so that every file
    holds the starting configuration's xyz, g(r), S(q), RMDF S(q) and (classical) the RMDF-updated
    force table, none of which depends on its unseeded generator; run twice with the append flags
    on, so that the files hold the running averages (count 2) and two xyz frames. (The executable's
    direct S(q) line, run.cpp:420-432, ends in a segmentation fault on these inputs whatever the run
    length; the direct S(q) file is pinned through the harness in sqd648 instead.)"""
    import subprocess
    from nnpengine_b200 import nnp_model as NM
    out = {}
    for mode in ("classical", "nnp_run"):
        d = os.path.join(work, mode)
        os.makedirs(d, exist_ok=True)
        s, table = cases.water_case()
        tpath, _ = rmdf_target(d)
        kw = dict(rmdf=(RMDF_STRENGTH, RMDF_GAMMA, tpath), steps=(0, 1, 1000, 1, 1), append=True)
        if mode == "classical":
            path, files = cases.write_run_input(d, mode, s, table, **kw)
        else:
            paths = cases.write_nnp_inputs(NM.gauss_model(), d)
            path, files = cases.write_run_input(d, mode, s, nnp_paths=paths, nbin=750, cutoffs=(6.0, 2.0, 6.0), **kw)
        for _ in range(2):
            subprocess.run([os.path.join(orc.REF_DIR, "nnp.exe"), mode, path], capture_output=True, text=True,
                           timeout=600, check=True)
        frames, types, box = cases.read_dump(files["xyz"])
        out[f"{mode}_xyz"] = frames
        out[f"{mode}_xyz_types"] = types
        out[f"{mode}_xyz_box"] = np.array(box)
        for k in ("gr", "sq", "sqd", "sqx", "force"):
            if os.path.exists(files[k]):
                num, rows = cases.read_dump(files[k])
                out[f"{mode}_{k}_num"] = num
                out[f"{mode}_{k}"] = rows
        print(f"dumps648 {mode}:", {k: out[f'{mode}_{k}'].shape for k in ("gr", "sq", "sqd", "sqx") if f'{mode}_{k}' in out})
    np.savez_compressed(os.path.join(HERE, "dumps648.npz"), **out)


def box648(work):
    """The 648-atom water box rescaled to other box lengths (positions times bl / 18.624, a smaller
    box and a larger one whose grid has more cells): the reference's snapshot at each, for the
    variable-box path (BL_MANAGER::setBL, run.cpp:688-712)."""
    s, table = cases.water_case()
    out = {}
    for tag, bl in (("small", 18.0), ("large", 25.0)):
        sb = cases.rescaled(s, bl)
        d = os.path.join(work, tag)
        f = cases.write_inputs(sb, table, d)
        v0 = os.path.join(d, "v0.bin")
        np.zeros((sb.natom, 3), np.float32).tofile(v0)
        snap = orc.run_ref_dump({"init": f["init"], "table": f"1000 {f['table']}", "cutoff": 10, "skin": 2,
                                 "gr_cutoff": 10, **bonded_cfg(), "velocity": v0, "mode": "snapshot"},
                                os.path.join(d, "snap"))
        counts, digests = cases.list_keys(snap["fulllist"], sb.natom)
        out.update({f"{tag}_bl": np.float64(bl), f"{tag}_x": sb.x, f"{tag}_list_counts": counts,
                    f"{tag}_list_digests": digests, f"{tag}_nghost": snap["info"]["nghost"],
                    f"{tag}_force": snap["force"].reshape(-1, 3)})
        print(f"box648 {tag}: bl {bl}, {int(counts.sum())} list entries, {snap['info']['nghost']} images")
    np.savez_compressed(os.path.join(HERE, "box648.npz"), **out)


ALL = [water648, mixture2000, nnp_gauss648, rmdf2000, driver648, sqd648, sqd2000, water3000, mixture30k, peroxide2048,
       dumps648, box648]

if __name__ == "__main__":
    names = sys.argv[1:]
    with tempfile.TemporaryDirectory() as t:
        for fn in ALL:
            if not names or fn.__name__ in names:
                fn(os.path.join(t, fn.__name__))
