"""Builds odevec_b200/libodevec_b200.so for sm_100a with nvcc.

One translation unit per (network variant, arithmetic mode) is compiled in
parallel:

* mode ``exact``: ``--fmad=false`` - no fused multiply-add, so every product
  and sum is rounded separately exactly as in the CPU oracle (G = 1 and 32,
  FP64 LU);
* mode ``fma``: ``--fmad=true`` (G = 1 and 32; FP64 LU and FP32 LU).

The kernel template is instantiated in a namespace named after the mode, so
the two modes never share a symbol.  The C-ABI layer (csrc/odevec_abi.cu) is
linked in with the CUDA runtime statically.  Rebuilds only what changed.
"""
from __future__ import annotations

import concurrent.futures as cf
import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "gen")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libodevec_b200.so")
ROOT = os.path.dirname(HERE)

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                 "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]
MODES = {"exact": ["--fmad=false"], "fma": ["--fmad=true"]}


def variants():
    reg = os.path.join(GEN, "registry.inc")
    if not os.path.exists(reg):
        return []
    return re.findall(r'OV_NET\((\w+), "([^"]+)"\)', open(reg).read())


PREC_CODE = {"fp64": 0, "fp64_fma": 1, "fp32_lu": 2}

# variant sets compiled into one multi-network kernel each (odevec_solve_many):
# the serving mix of ROBER, PRIMORDIAL and the 64-species network
MULTI_SETS = [("serving", ["rober_dense_none", "primordial_csc_ff", "syn64_csc_cmk"])]


def multi_sets():
    have = {cid for cid, _ in variants()}
    tags = dict(variants())
    return [(sid, cids, [tags[c] for c in cids]) for sid, cids in MULTI_SETS if all(c in have for c in cids)]


def write_multi_registry() -> str:
    """gen/multi.inc: OV_MULTI(sid, "TAG", ...) per compiled set"""
    lines = ["/* Generated by odevec_b200/build.py: the multi-network kernel sets. */"]
    for sid, _, tags in multi_sets():
        lines.append("OV_MULTI(%s, %s)" % (sid, ", ".join('"%s"' % t for t in tags)))
    path = os.path.join(GEN, "multi.inc")
    text = "\n".join(lines) + "\n"
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as fh:
            fh.write(text)
    return path


def write_tuning_table() -> str:
    """gen/tuning.inc: the autotuner's table (odevec_b200/tuning.json) as C,
    so the C ABI picks the tuned launch shape for options left at 0."""
    import json
    src = os.path.join(HERE, "tuning.json")
    table = json.load(open(src)) if os.path.exists(src) else {}
    lines = ["/* Generated by odevec_b200/build.py from odevec_b200/tuning.json -- do not edit.",
             "   OV_TUNE(tag, precision, group, device, staging, jac_batch, ss_batch, max_wait) */"]
    for key in sorted(table):
        net, prec, grp, dev = key.split("/")
        v = table[key]
        if prec not in PREC_CODE or '"' in dev or "\\" in dev:
            continue
        lines.append('OV_TUNE("%s", %d, %d, "%s", %d, %d, %d, %d)' % (
            net, PREC_CODE[prec], int(grp[1:]), dev, int(v["staging"]), int(v["jac_batch"]),
            int(v["ss_batch"]), int(v["max_wait"])))
    path = os.path.join(GEN, "tuning.inc")
    text = "\n".join(lines) + "\n"
    if not os.path.exists(path) or open(path).read() != text:
        with open(path, "w") as fh:
            fh.write(text)
    return path


def ensure_generated():
    if not variants():
        from . import shipped
        shipped.emit_all()


def _hash_files(paths, extra=""):
    h = hashlib.sha1(extra.encode())
    for p in sorted(paths):
        with open(p, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


def _headers():
    out = [os.path.join(ROOT, "include", "odevec_b200.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".h", ".cuh")):
            out.append(os.path.join(CSRC, f))
    return out


def _compile(src, obj, flags, log):
    cmd = [NVCC] + COMMON + flags + ["-Xptxas", "-v", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    with open(log, "w") as fh:
        fh.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stderr[-4000:]))
    return obj


def build(force: bool = False, jobs: int = 0, verbose: bool = False) -> str:
    ensure_generated()
    os.makedirs(BUILD, exist_ok=True)
    hdrs = _headers()
    tasks = []
    objs = []
    for cid, tag in variants():
        for mode, flags in MODES.items():
            src = os.path.join(BUILD, "kernels_%s_%s.cu" % (cid, mode))
            text = ("/* generated by odevec_b200/build.py */\n#define OV_MODE_NS %s\n"
                    '#include "bdf_kernel.cuh"\n#include "gen/net_%s.cuh"\n'
                    "OV_DEFINE_LAUNCHER(%s, %d)\n" % (mode, cid, cid, 1 if mode == "fma" else 0))
            if not os.path.exists(src) or open(src).read() != text:
                with open(src, "w") as fh:
                    fh.write(text)
            deps = hdrs + [os.path.join(GEN, "net_%s.h" % cid), os.path.join(GEN, "net_%s.cuh" % cid)]
            key = _hash_files(deps + [src], " ".join(COMMON + flags))
            obj = os.path.join(BUILD, "kernels_%s_%s.o" % (cid, mode))
            stamp = obj + ".key"
            objs.append(obj)
            if force or not os.path.exists(obj) or not os.path.exists(stamp) or open(stamp).read() != key:
                tasks.append((src, obj, flags, obj + ".log", stamp, key))
    for sid, cids, _ in multi_sets():
        for mode, flags in MODES.items():
            src = os.path.join(BUILD, "multi_%s_%s.cu" % (sid, mode))
            text = ("/* generated by odevec_b200/build.py */\n#define OV_MODE_NS %s\n"
                    '#include "bdf_kernel.cuh"\n' % mode
                    + "".join('#include "gen/net_%s.cuh"\n' % c for c in cids)
                    + "OV_DEFINE_MULTI(%s, %d, %s)\n" % (sid, 1 if mode == "fma" else 0,
                                                        ", ".join("ov_net_%s" % c for c in cids)))
            if not os.path.exists(src) or open(src).read() != text:
                with open(src, "w") as fh:
                    fh.write(text)
            deps = hdrs + [os.path.join(GEN, "net_%s.%s" % (c, ext)) for c in cids for ext in ("h", "cuh")]
            key = _hash_files(deps + [src], " ".join(COMMON + flags))
            obj = os.path.join(BUILD, "multi_%s_%s.o" % (sid, mode))
            stamp = obj + ".key"
            objs.append(obj)
            if force or not os.path.exists(obj) or not os.path.exists(stamp) or open(stamp).read() != key:
                tasks.append((src, obj, flags, obj + ".log", stamp, key))
    probe_src = os.path.join(CSRC, "ov_probe.cu")
    probe_obj = os.path.join(BUILD, "ov_probe.o")
    pkey = _hash_files(hdrs + [probe_src], " ".join(COMMON))
    if force or not os.path.exists(probe_obj) or not os.path.exists(probe_obj + ".key") or \
            open(probe_obj + ".key").read() != pkey:
        tasks.append((probe_src, probe_obj, ["--fmad=true"], probe_obj + ".log", probe_obj + ".key", pkey))
    objs.append(probe_obj)
    abi_src = os.path.join(CSRC, "odevec_abi.cu")
    abi_obj = os.path.join(BUILD, "odevec_abi.o")
    tune_inc = write_tuning_table()
    multi_inc = write_multi_registry()
    key = _hash_files(hdrs + [abi_src, os.path.join(GEN, "registry.inc"),
                              os.path.join(GEN, "includes_c.inc"), tune_inc, multi_inc] +
                      [os.path.join(GEN, "net_%s.h" % c) for c, _ in variants()], " ".join(COMMON))
    if force or not os.path.exists(abi_obj) or not os.path.exists(abi_obj + ".key") or \
            open(abi_obj + ".key").read() != key:
        tasks.append((abi_src, abi_obj, [], abi_obj + ".log", abi_obj + ".key", key))
    objs.append(abi_obj)
    if tasks:
        n = jobs or min(len(tasks), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(n) as ex:
            futs = {ex.submit(_compile, s, o, f, lg): (o, st, k) for s, o, f, lg, st, k in tasks}
            for fu in cf.as_completed(futs):
                fu.result()
                o, st, k = futs[fu]
                with open(st, "w") as fh:
                    fh.write(k)
                if verbose:
                    print("compiled", os.path.basename(o))
    if tasks or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB + ".tmp"] + objs
        subprocess.run(cmd, check=True)
        os.replace(LIB + ".tmp", LIB)
    return LIB


def ptxas_report():
    """Registers / spills per kernel from the last build's ptxas output."""
    out = []
    for f in sorted(os.listdir(BUILD)):
        if f.endswith(".log"):
            txt = open(os.path.join(BUILD, f)).read()
            for m in re.finditer(r"Compiling entry function '(\S+)'.*?\n(.*?Used (\d+) registers[^\n]*)",
                                 txt, re.S):
                name = m.group(1)
                info = m.group(2)
                spill = re.search(r"(\d+) bytes spill stores, (\d+) bytes spill loads", info)
                stack = re.search(r"(\d+) bytes stack frame", info)
                out.append((f, name, int(m.group(3)), stack.group(1) if stack else "?",
                            spill.groups() if spill else ("?", "?")))
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    if "--report" in sys.argv:
        for r in ptxas_report():
            print(r)
