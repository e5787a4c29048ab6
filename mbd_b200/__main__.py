"""Command line of the engine: the pmbd.x front end and its input tooling.

    python -m mbd_b200 run geometry.in [setting.in] [--mode plain|mixed|mixed_learned]
                       [--network FILE] [--device N]
        The MBD@rsSCS energy of one geometry on the GPU, printed as the MBD
        section of pmbd.x's report (MBD_rsSCS.f90:59-60 takes the same two
        files; the report fields are UTILS.f90:223-331).  Exit status 1 with
        the engine's message when the geometry fails (unknown element,
        non-positive-definite relay matrix, ...).
    python -m mbd_b200 tile geometry.in N1 N2 N3 [-o out.in]
        Supercell of a periodic geometry, N1 x N2 x N3 copies along its three
        lattice vectors (examples/process.py tiles the graphene cell along
        two of them); written to out.in or stdout.
    python -m mbd_b200 generate cluster|box|sheet|benzene|batch [--atoms N] [--seed S]
                       [--reps R] [--count C] [--scs-cut A] [--cfdm-cut A] [--sc-cut A]
                       -o geometry.in [--settings setting.in]
        Seeded synthetic inputs in pmbd.x's formats, the shapes the benchmarks
        and tests use: an isolated {H,C,N,O} cluster of N atoms at molecular
        density, a periodic box of N atoms (cut-offs in Angstrom, default
        120/100/25), a graphene sheet of R x R cells (vacuum along z),
        benzene, or a batch of C clusters of 20-600 atoms (-o is then a
        directory that receives geometry_<k>.in and setting.in).
    python -m mbd_b200 train --out net.bin [--geoms 160] [--epochs 12] [--boxes]
        Trains the learned warm start's network on the GPU on seeded synthetic
        clusters (or periodic boxes) of 50-400 atoms and writes the
        checkpoint (versioned, SHA-256-checked) that `run --network` loads.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

from .io import InputError, format_report, parse_geometry, parse_settings, tile, write_geometry, write_settings


def _run(args) -> int:
    from .engine import Engine, strerror
    with open(args.geometry) as fh:
        geo = parse_geometry(fh.read())
    st_text = ""
    if args.settings:
        with open(args.settings) as fh:
            st_text = fh.read()
    st = parse_settings(st_text)
    with Engine(args.device) as eng:
        if args.mode == "mixed_learned":
            if args.network:
                eng.load_network(args.network)
            else:
                eng.use_network(False)     # block-CG from zero: the method without the network
        res = eng.energy(geo, st, mode=args.mode, check=False)
    if res.status != 0:
        print(f"mbd_b200: {strerror(res.status)} (status {res.status})", file=sys.stderr)
        return 1
    print(format_report(geo, res))
    return 0


def _tile(args) -> int:
    with open(args.geometry) as fh:
        geo = parse_geometry(fh.read())
    text = write_geometry(tile(geo, (args.n1, args.n2, args.n3)))
    if args.out:
        with open(args.out, "w") as fh:
            fh.write(text)
    else:
        sys.stdout.write(text)
    return 0


def _generate(args) -> int:
    import os

    from . import synthetic as sy
    if args.kind == "batch":
        os.makedirs(args.out, exist_ok=True)
        items = sy.cluster_batch(count=args.count, seed=args.seed)
        for k, (geo, _) in enumerate(items):
            with open(os.path.join(args.out, f"geometry_{k}.in"), "w") as fh:
                fh.write(write_geometry(geo))
        with open(os.path.join(args.out, "setting.in"), "w") as fh:
            fh.write(write_settings(items[0][1]))
        return 0
    if args.kind in ("cluster", "box") and (args.atoms is None or args.atoms < 1):
        raise InputError(f"generate {args.kind}: --atoms N (>= 1) is required")
    if args.kind == "cluster":
        geo, st = sy.cluster(args.atoms, seed=args.seed)
    elif args.kind == "box":
        geo, st = sy.periodic_box(args.atoms, seed=args.seed, scs_cut=args.scs_cut, cfdm_cut=args.cfdm_cut,
                                  sc_cut=args.sc_cut)
    elif args.kind == "sheet":
        geo, st = sy.graphene_sheet(args.reps)
    else:
        geo, st = sy.benzene()
    with open(args.out, "w") as fh:
        fh.write(write_geometry(geo))
    if args.settings:
        with open(args.settings, "w") as fh:
            fh.write(write_settings(st))
    return 0


def _train(args) -> int:
    from . import synthetic as sy
    from .engine import Engine
    rng = np.random.default_rng(args.seed)
    gen = sy.periodic_box if args.boxes else sy.cluster
    items = [gen(int(n), seed=100000 + k) for k, n in enumerate(rng.integers(50, 401, size=args.geoms))]
    with Engine(args.device) as eng:
        loss = eng.learned_train([g for g, _ in items], [s for _, s in items], epochs=args.epochs, lr=args.lr,
                                 seed=args.seed)
        eng.save_network(args.out)
    print(f"trained on {len(items)} {'boxes' if args.boxes else 'clusters'}: loss {loss[0]:.4g} -> {loss[-1]:.4g}; "
          f"wrote {args.out}")
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m mbd_b200", description=__doc__.split("\n\n")[0])
    sub = ap.add_subparsers(dest="cmd", required=True)
    r = sub.add_parser("run", help="MBD@rsSCS energy of one geometry, pmbd.x report")
    r.add_argument("geometry")
    r.add_argument("settings", nargs="?")
    r.add_argument("--mode", default="plain", choices=["plain", "mixed", "mixed_learned"])
    r.add_argument("--network", default=None, help="network checkpoint for --mode mixed_learned")
    r.add_argument("--device", type=int, default=0)
    t = sub.add_parser("tile", help="supercell of a periodic geometry")
    t.add_argument("geometry")
    t.add_argument("n1", type=int)
    t.add_argument("n2", type=int)
    t.add_argument("n3", type=int)
    t.add_argument("-o", "--out", default=None)
    gsub = sub.add_parser("generate", help="seeded synthetic geometry (and settings) in pmbd.x's formats")
    gsub.add_argument("kind", choices=["cluster", "box", "sheet", "benzene", "batch"])
    gsub.add_argument("--atoms", type=int, default=None)
    gsub.add_argument("--seed", type=int, default=0)
    gsub.add_argument("--reps", type=int, default=8, help="sheet: cells along each in-plane vector")
    gsub.add_argument("--count", type=int, default=256, help="batch: number of clusters")
    gsub.add_argument("--scs-cut", type=float, default=120.0)
    gsub.add_argument("--cfdm-cut", type=float, default=100.0)
    gsub.add_argument("--sc-cut", type=float, default=25.0)
    gsub.add_argument("-o", "--out", required=True)
    gsub.add_argument("--settings", default=None, help="also write the matching setting.in here")
    n = sub.add_parser("train", help="train the learned warm start and write a checkpoint")
    n.add_argument("--out", required=True)
    n.add_argument("--geoms", type=int, default=160)
    n.add_argument("--epochs", type=int, default=12)
    n.add_argument("--lr", type=float, default=1e-3)
    n.add_argument("--seed", type=int, default=7)
    n.add_argument("--boxes", action="store_true", help="periodic boxes instead of isolated clusters")
    n.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    try:
        return {"run": _run, "tile": _tile, "generate": _generate, "train": _train}[args.cmd](args)
    except InputError as exc:
        print(f"mbd_b200: {exc}", file=sys.stderr)
        return 1


if __name__ == "__main__":
    sys.exit(main())
