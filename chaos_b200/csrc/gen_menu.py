"""Generate the compiled menu of orbit-kernel instances (cl_menu_*.cu).

Each entry is (system kind, d, precision, frames); a frame is (k, reducer tokens). The key string is the one
`cl::run_key` builds from a cl_run, so a run finds its instance by lookup; the C++ types are the kernel's template
arguments. Run as a build step (chaos_b200/build.py calls it); the output is deterministic.
"""
from __future__ import annotations

import os

HERE = os.path.dirname(os.path.abspath(__file__))

SYS_STANDARD, SYS_WRAPPED, SYS_FROESCHLE, SYS_CHAIN, SYS_LINEAR, SYS_HH, SYS_SPLIT = 1, 2, 3, 4, 5, 6, 7
SYS_WRAPPED_FRO, SYS_WRAPPED_CHAIN = 8, 9
QR = [f"QR{a}" for a in range(1, 7)]   # CGS, MGS, RGS, Householder, augmented, Givens


def red_type(tokens):
    """C++ reducer types of a frame's token list ("GALI","SALI" adjacent is the fused GALI+SALI state)."""
    out, i = [], 0
    while i < len(tokens):
        t = tokens[i]
        if t == "GALI" and i + 1 < len(tokens) and tokens[i + 1] == "SALI":
            out.append("RGALI<true>")
            i += 2
            continue
        if t.startswith("QR"):
            out.append(f"RQR<{int(t[2:])}>")
        elif t == "BEN":
            out.append("RBenettin")
        elif t == "SALI":
            out.append("RSALI")
        elif t == "GALI":
            out.append("RGALI<false>")
        elif t.startswith("MEGNO"):
            out.append(f"RMEGNO<{'true' if t[5:] == '1' else 'false'}>")
        elif t.startswith("FLI"):
            out.append(f"RFLI<{'true' if t[3:] == '1' else 'false'}>")
        else:
            raise ValueError(t)
        i += 1
    return out


def sys_type(kind, d):
    return {SYS_STANDARD: "SysStandard", SYS_WRAPPED: "SysWrapped", SYS_FROESCHLE: "SysFroeschle",
            SYS_CHAIN: f"SysChain<{d // 2}>", SYS_LINEAR: f"SysLinear<{d}>", SYS_HH: "SysGauss3HH",
            SYS_SPLIT: "SysSplitHH", SYS_WRAPPED_FRO: "SysWrappedFroeschle",
            SYS_WRAPPED_CHAIN: f"SysWrappedChain<{d // 2}>"}[kind]


def key(kind, d, prec, frames):
    return f"s{kind}d{d}p{prec}|" + "".join(f"k{k}:{','.join(t)}|" for k, t in frames)


def menu():
    """The compiled menu, grouped into translation units (compiled in parallel)."""
    groups: dict[str, list] = {}

    def add(group, kind, d, prec, frames, minbs=(1,)):
        groups.setdefault(group, []).append((kind, d, prec, frames, minbs))

    k2_chains = [[q] for q in QR] + [["SALI"], ["GALI"], ["MEGNO1"], ["FLI1"], ["MEGNO0", "FLI0", "QR6"],
                                     ["MEGNO0", "SALI"], ["FLI0", "SALI"], ["MEGNO0", "FLI0", "SALI"], []]
    k1_chains = [["BEN"]] + [[q] for q in QR]
    for kind, g in ((SYS_STANDARD, "std"), (SYS_WRAPPED, "wrapped")):
        for ch in k1_chains:
            add(g, kind, 2, 0, [(1, ch)])
        for ch in k2_chains:
            add(g, kind, 2, 0, [(2, ch)])
        for ch in (["QR2"], ["QR4"], ["QR6"]):
            add(g + "_mixed", kind, 2, 1, [(2, ch)])
        add(g + "_mixed", kind, 2, 1, [(1, ["BEN"])])
    # linear symplectic maps: the reference's known-answer fixtures
    for ch in k1_chains:
        add("linear", SYS_LINEAR, 2, 0, [(1, ch)])
    for ch in k2_chains:
        add("linear", SYS_LINEAR, 2, 0, [(2, ch)])
    for k in (2, 4):
        for ch in [[q] for q in QR] + [["GALI"]]:
            add("linear4", SYS_LINEAR, 4, 0, [(k, ch)])
    add("linear4", SYS_LINEAR, 4, 0, [(1, ["BEN"])])
    for ch in (["QR2"], ["QR4"], ["GALI"]):
        add("linear6", SYS_LINEAR, 6, 0, [(6, ch)])
    # Froeschle (4D coupled standard maps)
    for ch in k1_chains:
        add("fro", SYS_FROESCHLE, 4, 0, [(1, ch)])
    for ch in k2_chains:
        add("fro", SYS_FROESCHLE, 4, 0, [(2, ch)])
    for k in (3, 4):
        for ch in [[q] for q in QR] + [["GALI"]]:
            add("fro4", SYS_FROESCHLE, 4, 0, [(k, ch)])
    add("fro4", SYS_FROESCHLE, 4, 0, [(4, ["GALI", "SALI"])])
    # the fused QRSpectrum + GALI_4 + SALI ensemble (two frames, one orbit) in both precisions
    for prec in (0, 1):
        add("fro_fused" if prec == 0 else "fro_mixed", SYS_FROESCHLE, 4, prec, [(4, ["QR4"]), (4, ["GALI", "SALI"])],
            minbs=(1, 2, 3) if prec == 0 else (1, 2, 3, 4))
    for ch in (["QR4"], ["QR2"], ["GALI", "SALI"], ["GALI"]):
        add("fro_mixed", SYS_FROESCHLE, 4, 1, [(4, ch)])
    for ch in (["QR2"], ["SALI"], ["MEGNO1"], ["MEGNO0", "SALI"]):
        add("fro_mixed", SYS_FROESCHLE, 4, 1, [(2, ch)])
    # the same map on the torus with winding counts (the C2 ensemble's coordinates in [0, 2 pi)^4)
    for ch in k1_chains[:3]:
        add("wfro", SYS_WRAPPED_FRO, 4, 0, [(1, ch)])
    for ch in (["QR2"], ["QR6"], ["SALI"], ["MEGNO1"], ["FLI1"], ["MEGNO0", "FLI0", "QR6"], ["MEGNO0", "SALI"]):
        add("wfro", SYS_WRAPPED_FRO, 4, 0, [(2, ch)])
    for ch in (["QR4"], ["QR2"], ["GALI"], ["GALI", "SALI"]):
        add("wfro", SYS_WRAPPED_FRO, 4, 0, [(4, ch)])
    for prec in (0, 1):
        add("wfro" if prec == 0 else "wfro_mixed", SYS_WRAPPED_FRO, 4, prec, [(4, ["QR4"]), (4, ["GALI", "SALI"])],
            minbs=(1, 2, 3) if prec == 0 else (1, 2, 3, 4))
    for ch in (["QR4"], ["GALI", "SALI"]):
        add("wfro_mixed", SYS_WRAPPED_FRO, 4, 1, [(4, ch)])
    add("wfro_mixed", SYS_WRAPPED_FRO, 4, 1, [(2, ["QR2"])])
    # coupled standard-map lattices, N = 2..8 sites
    for N in range(2, 9):
        d = 2 * N
        kk = min(d, 8)
        g = f"chain{N}"
        for prec in (0, 1):
            for ch in (["QR2"], ["QR4"], ["GALI"]):
                add(g, SYS_CHAIN, d, prec, [(kk, ch)])
            for ch in (["QR2"], ["SALI"], ["MEGNO1"]):
                add(g, SYS_CHAIN, d, prec, [(2, ch)])
        add(g, SYS_CHAIN, d, 0, [(1, ["BEN"])])
        # the lattice on the torus with winding counts
        for prec in (0, 1):
            for ch in (["QR2"], ["QR4"], ["GALI"]):
                add("w" + g, SYS_WRAPPED_CHAIN, d, prec, [(kk, ch)])
        for ch in (["QR2"], ["SALI"], ["MEGNO1"]):
            add("w" + g, SYS_WRAPPED_CHAIN, d, 0, [(2, ch)])
        add("w" + g, SYS_WRAPPED_CHAIN, d, 0, [(1, ["BEN"])])
    # IntegratorMap(Gauss(Float64, 3), HenonHeilesFlow(), dt)
    for ch in (["MEGNO0", "FLI0", "QR6"], ["QR2"], ["QR6"], ["MEGNO1"], ["FLI1"], ["SALI"], ["GALI"]):
        add("hh", SYS_HH, 4, 0, [(2, ch)])
    for ch in (["QR2"], ["QR4"], ["GALI"]):
        add("hh", SYS_HH, 4, 0, [(4, ch)])
    add("hh", SYS_HH, 4, 0, [(1, ["BEN"])])
    add("hh_mixed", SYS_HH, 4, 1, [(2, ["MEGNO0", "FLI0", "QR6"])])
    add("hh_mixed", SYS_HH, 4, 1, [(2, ["QR2"])])
    # the same in the mixed kernels (Float64 orbit and stage states, Float32 tangent)
    for ch, k in ((["MEGNO0", "FLI0", "QR6"], 2), (["QR2"], 2), (["QR4"], 4), (["GALI"], 4)):
        add("split_mixed", SYS_SPLIT, 4, 1, [(k, ch)], minbs=(1, 2, 3, 4))
    # IntegratorMap(SplittingMethod(c, d), HenonHeilesFlow(), dt): any table of at most CL_MAX_STAGES (128) stages
    for ch in (["MEGNO0", "FLI0", "QR6"], ["QR2"], ["QR6"], ["MEGNO1"], ["FLI1"], ["SALI"], ["GALI"]):
        add("split", SYS_SPLIT, 4, 0, [(2, ch)])
    for ch in (["QR2"], ["QR4"], ["GALI"]):
        add("split", SYS_SPLIT, 4, 0, [(4, ch)])
    add("split", SYS_SPLIT, 4, 0, [(1, ["BEN"])])
    return groups


# The batched uneven ensemble: (system kind, d, precision, k, chain, tau unrolled in the variants).
ENSEMBLE = [(SYS_STANDARD, 2, p, 2, ["QR4"], 5) for p in (0, 1)] + \
           [(SYS_CHAIN, 4, p, 4, ["QR4"], 10) for p in (0, 1)] + \
           [(SYS_CHAIN, 8, p, 8, ["QR4"], 10) for p in (0, 1)] + \
           [(SYS_CHAIN, 16, p, 8, ["QR4"], 20) for p in (0, 1)]


def render_ensemble(entries):
    out = ['// Generated by chaos_b200/csrc/gen_menu.py (do not edit): ensemble kernel instances.',
           '#include "cl_coop.cuh"', '', 'namespace cl {', 'namespace {']
    for idx, (kind, d, prec, k, ch, U) in enumerate(entries):
        real = "double" if prec == 0 else "float"
        ft = f"Frame<{k}{''.join(', ' + t for t in red_type(ch))}>"
        out.append(f"cudaError_t E{idx}(const cl_run& r, const EArgs& a, int g, const ETune& t, cudaStream_t s, LaunchInfo* i) {{\n"
                   f"    return launch_ensemble_any<{sys_type(kind, d)}, {real}, {ft}, {U}>(r, a, g, t, s, i);\n}}\n"
                   f"const ERegistrar R{idx}(\"{key(kind, d, prec, [(k, ch)])}\", E{idx});")
    out += ['}  // namespace', '}  // namespace cl', '']
    return "\n".join(out)


HEADER = """// Generated by chaos_b200/csrc/gen_menu.py (do not edit): compiled orbit-kernel instances, group "{group}".
#include "cl_registry.cuh"
{extra}
namespace cl {{
namespace {{
"""


def coop(kind, d, frames):
    """Lattices with d >= 8 and one frame run `propagate` cooperatively (cl_coop_orbit.cuh) by default."""
    return kind == SYS_CHAIN and d >= 8 and len(frames) == 1


def render(group, entries):
    extra = ('#include "cl_gauss.cuh"\n' if any(e[0] == SYS_HH for e in entries) else "") + \
            ('#include "cl_split.cuh"\n' if any(e[0] == SYS_SPLIT for e in entries) else "") + \
            ('#include "cl_coop_orbit.cuh"\n' if any(coop(e[0], e[1], e[3]) for e in entries) else "")
    out = [HEADER.format(group=group, extra=extra)]
    for idx, (kind, d, prec, frames, minbs) in enumerate(entries):
        real = "double" if prec == 0 else "float"
        ftypes = [f"Frame<{k}{''.join(', ' + t for t in red_type(ch))}>" for k, ch in frames]
        if coop(kind, d, frames):   # variant V_COOP (the default) and the one-thread kernel as variant 1
            out.append(f"cudaError_t L{idx}(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {{\n"
                       f"    return launch_chain_instance<{d // 2}, {real}, {ftypes[0]}>(r, a, A, s, i, m);\n}}\n"
                       f"const Registrar R{idx}(\"{key(kind, d, prec, frames)}\", L{idx}, minb_mask<1>() | (1u << (V_COOP - 1)));\n")
            continue
        while len(ftypes) < 3:
            ftypes.append("NoFrame")
        mb = ", ".join(str(m) for m in minbs)
        out.append(f"cudaError_t L{idx}(const cl_run& r, const KArgs& a, const double* A, cudaStream_t s, LaunchInfo* i, int m) {{\n"
                   f"    return launch_instance<{sys_type(kind, d)}, {real}, {', '.join(ftypes)}, {len(frames)}, {mb}>(r, a, A, s, i, m);\n}}\n"
                   f"const Registrar R{idx}(\"{key(kind, d, prec, frames)}\", L{idx}, minb_mask<{mb}>());\n")
    out.append("}  // namespace\n}  // namespace cl\n")
    return "\n".join(out)


def main():
    groups = menu()
    written = []
    for g, entries in groups.items():
        path = os.path.join(HERE, f"cl_menu_{g}.cu")
        text = render(g, entries)
        old = open(path).read() if os.path.exists(path) else None
        if old != text:
            with open(path, "w") as f:
                f.write(text)
        written.append(path)
    for prec in (0, 1):
        path = os.path.join(HERE, f"cl_ens_menu_p{prec}.cu")
        text = render_ensemble([e for e in ENSEMBLE if e[2] == prec])
        if (open(path).read() if os.path.exists(path) else None) != text:
            with open(path, "w") as f:
                f.write(text)
        written.append(path)
    for fn in os.listdir(HERE):   # drop stale groups
        if fn.startswith(("cl_menu_", "cl_ens_menu_")) and fn.endswith(".cu") and os.path.join(HERE, fn) not in written:
            os.remove(os.path.join(HERE, fn))
    return written


if __name__ == "__main__":
    for p in main():
        print(p)
