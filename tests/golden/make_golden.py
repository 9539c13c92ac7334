"""Generates the golden fixtures in this directory from the reference
MGBrain itself (oracle/_ref, built by `make -C oracle ref`).

  python tests/golden/make_golden.py net   [--out DIR]
      runs the reference's gen_net (oracle/_ref/ref_gen, CPU) on each case's
      model description -> <case>.net, plus <case>.v0 (seeded initial V).
  python tests/golden/make_golden.py sim   [--out DIR]
      runs the reference kernels (oracle/_ref/ref_sim, sm_100a build with
      --fmad=false; needs a GPU) for each case -> <case>.ref.raster,
      <case>.ref.state, and MGSimulator::simulate itself for the cases
      flagged `simulate` -> <case>.sim.state.

cases.json records every seed and step count used.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
import mgb_testlib as T  # noqa: E402


def lif_line(dt, v_init, v_reset, v_th, t_ref, leak=0.0):
    c = [0.0] * 30
    c[0], c[1], c[3], c[4], c[8], c[9] = dt, v_init, v_reset, v_th, t_ref, leak
    return "lifconst " + " ".join(repr(float(np.float32(x))) for x in c)


CASES = {
    # Brunel C0 scaled to 600 neurons: LIFB E/I + POISSON, one 15-step delay,
    # seeded V0 ~ U[0, 20 mV); J raised so that a small network stays active.
    "c0s": dict(
        spec="\n".join([
            "timestep 0.0001",
            lif_line(0.0001, 0.0, 0.01, 0.02, 0.002),
            "pop 400 LIFB 0", "pop 100 LIFB 0", "pop 100 POISSON 1",
            "conn 2 0 0.0005 0.0005 0.0015 0.0015 0.1 STATIC",
            "conn 2 1 0.0005 0.0005 0.0015 0.0015 0.1 STATIC",
            "conn 0 0 0.0005 0.0005 0.0015 0.0015 0.1 STATIC",
            "conn 0 1 0.0005 0.0005 0.0015 0.0015 0.1 STATIC",
            "conn 1 0 -0.0025 -0.0025 0.0015 0.0015 0.1 STATIC",
            "conn 1 1 -0.0025 -0.0025 0.0015 0.0015 0.1 STATIC",
            "rate 2 0.02", ""]),
        mt=11, rnd=3, seed=101, steps=2000, v0=(0.0, 0.02, 7), stdp=0, simulate=0.2),
    # the reference's own Brunel maker at 20k synapses (V starts at V_init=0)
    "brunel_maker": dict(spec="timestep 0.0001\nmaker brunel 20000\nrate 0 0.002\n",
                         mt=5, rnd=5, seed=202, steps=2000, v0=None, stdp=0, simulate=0.2),
    # the reference's Vogels maker: LIFE neurons, no external input
    "vogel_maker": dict(spec="timestep 0.0001\nmaker vogel 20000\n",
                        mt=6, rnd=6, seed=303, steps=2000, v0=(-0.06, -0.05, 8), stdp=0),
    # exponential LIF (ConstGen::gen_life_const) with delays drawn 1.0..3.0 ms
    "lif_mixed": dict(
        spec="\n".join([
            "timestep 0.0001",
            "life_const 0.0 0.0 0.0 0.0 0.02 0.001 0.005 0.005 0.01 0.0",
            "pop 300 LIF 0", "pop 80 LIF 0", "pop 120 POISSON 1",
            "conn 2 0 0.002 0.002 0.001 0.003 0.2 STATIC",
            "conn 2 1 0.002 0.002 0.001 0.003 0.2 STATIC",
            "conn 0 0 0.0008 0.0008 0.001 0.003 0.1 STATIC",
            "conn 0 1 0.0008 0.0008 0.001 0.003 0.1 STATIC",
            "conn 1 0 -0.004 -0.004 0.001 0.002 0.1 STATIC",
            "rate 2 0.01", ""]),
        mt=7, rnd=7, seed=404, steps=2000, v0=None, stdp=0),
    # Vogels-Abbott C1 scaled: LIFB shifted by +60 mV (V_th 10 mV, reset 0,
    # t_ref 5 ms), 1-step delays, a 20-neuron one-to-one Poisson kick for
    # the first 500 steps
    "c1s": dict(
        spec="\n".join([
            "timestep 0.0001",
            lif_line(0.0001, 0.0, 0.0, 0.01, 0.005),
            "pop 20 LIFB 0", "pop 380 LIFB 0", "pop 100 LIFB 0", "pop 20 POISSON 1",
            "conn 3 0 0.02 0.02 0.0001 0.0001 0 STATIC",
            "conn 0 0 0.00027 0.00027 0.0001 0.0001 0.08 STATIC",
            "conn 0 1 0.00027 0.00027 0.0001 0.0001 0.08 STATIC",
            "conn 0 2 0.00027 0.00027 0.0001 0.0001 0.08 STATIC",
            "conn 1 0 0.00027 0.00027 0.0001 0.0001 0.08 STATIC",
            "conn 1 1 0.00027 0.00027 0.0001 0.0001 0.08 STATIC",
            "conn 1 2 0.00027 0.00027 0.0001 0.0001 0.08 STATIC",
            "conn 2 0 -0.0045 -0.0045 0.0001 0.0001 0.08 STATIC",
            "conn 2 1 -0.0045 -0.0045 0.0001 0.0001 0.08 STATIC",
            "conn 2 2 -0.0045 -0.0045 0.0001 0.0001 0.08 STATIC",
            "rate 3 0.01", ""]),
        mt=8, rnd=8, seed=505, steps=2000, v0=(0.0, 0.01, 9), stdp=0, rates_off=500),
    # global STDP (Config::STDP) on a small LIFB network
    "stdp_small": dict(
        spec="\n".join([
            "timestep 0.0001",
            lif_line(0.0001, 0.0, 0.0, 0.02, 0.002),
            "stdpconst 0.0001 -0.000105 40 40 0.01 0.0",
            "pop 60 POISSON 1", "pop 160 LIFB 0",
            "conn 0 1 0.004 0.004 0.0001 0.0001 0.3 STATIC",
            "conn 1 1 0.001 0.001 0.0005 0.0005 0.05 STATIC",
            "rate 0 0.01", ""]),
        mt=9, rnd=9, seed=606, steps=2000, v0=None, stdp=1),
}


def v0_for(case, n):
    if case["v0"] is None:
        return None
    lo, hi, s = case["v0"]
    return np.random.default_rng(s).uniform(lo, hi, n).astype(np.float32)


def cmd_net(out):
    os.makedirs(out, exist_ok=True)
    manifest = {}
    for name, c in CASES.items():
        net = T.ref_gen(c["spec"], c["mt"], c["rnd"], os.path.join(out, name + ".net"))
        os.remove(os.path.join(out, name + ".net.spec"))
        with open(os.path.join(out, name + ".spec"), "w") as f:
            f.write(c["spec"])
        v0 = v0_for(c, net["n"])
        if v0 is not None:
            v0.tofile(os.path.join(out, name + ".v0"))
        manifest[name] = {k: v for k, v in c.items() if k != "spec"}
        manifest[name].update(n=int(net["n"]), S=int(len(net["src"])))
        print(name, net["n"], len(net["src"]))
    with open(os.path.join(out, "cases.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)


def cmd_sim(src_dir, out):
    os.makedirs(out, exist_ok=True)
    man = json.load(open(os.path.join(src_dir, "cases.json")))
    for name, c in man.items():
        net = os.path.join(src_dir, name + ".net")
        v0 = os.path.join(src_dir, name + ".v0")
        v0 = v0 if os.path.exists(v0) else "-"
        env = dict(os.environ, MGB_REF_SEED=str(c["seed"]))
        args = [T.REF_SIM, "steps", net, os.path.join(out, name + ".ref"), str(c["steps"]), v0,
                str(c["stdp"])]
        if c.get("rates_off") is not None:
            args.append(str(c["rates_off"]))
        r = subprocess.run(args, env=env, capture_output=True, text=True)
        print(name, r.stdout.strip(), r.stderr.strip()[-300:])
        r.check_returncode()
        if c.get("simulate"):
            args = [T.REF_SIM, "simulate", net, os.path.join(out, name + ".sim"), str(c["simulate"]), v0,
                    str(c["stdp"])]
            r = subprocess.run(args, env=env, capture_output=True, text=True)
            print(name, "simulate", r.stdout.strip()[-200:])
            r.check_returncode()


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["net", "sim"])
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--src", default=HERE)
    a = ap.parse_args()
    if a.what == "net":
        cmd_net(a.out)
    else:
        cmd_sim(a.src, a.out)
