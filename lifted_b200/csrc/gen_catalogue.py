#!/usr/bin/env python3
"""Generates wavelet_catalogue.inc, the lifting-step table of the 34
predefined wavelets, from the reference's catalogue header.

The table has to hold exactly the reference's factorisations: the same step
kinds, offsets and tap counts, and the coefficient literals spelled exactly
as written (suffix included), so that casting them to float/double gives the
same constants as the reference's ``static_cast<T>(literal)``
(src/lifted-common.hpp:998-1032) and ``(T)(1.0L / c)`` for scale steps
(src/lifted-common.hpp:951-963).  Known typos in the literals are kept
(Bior2_6 -0.076171874L, Bior4_4 0.226562L, Symlet4's last literal without an
``L`` suffix).

Usage: python gen_catalogue.py [path/to/lifted/src] > wavelet_catalogue.inc
(default: $LIFTED_REFERENCE/src, else the src/ of a checkout named
"reference" beside this repository).  The generated file is committed; this
script only reruns when the catalogue changes.
"""
import os
import re
import sys
from pathlib import Path

STEP_RE = re.compile(
    r"constexpr\s+static\s+auto\s+(\w+)\s*=\s*(?:detail::)?"
    r"(update_s|update_d|unit_update_s|unit_update_d|repeat_update_s|"
    r"repeat_update_d|ScaleStep)\s*<\s*T\s*(?:,\s*([^>]+?))?\s*>\s*\((.*?)\)\s*;",
    re.S,
)
CLASS_RE = re.compile(r"class\s+(\w+)\s*\{(.*?)\n\s*\};", re.S)
ENUM_RE = re.compile(r"X\((\w+),\s*(\d+)\)")


def strip_comments(text: str) -> str:
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def split_args(args: str):
    return [a.strip() for a in args.replace("\n", " ").split(",") if a.strip()]


def main() -> None:
    if len(sys.argv) > 1:
        src = Path(sys.argv[1])
    elif os.environ.get("LIFTED_REFERENCE"):
        src = Path(os.environ["LIFTED_REFERENCE"]) / "src"
    else:
        src = Path(__file__).resolve().parents[3] / "reference" / "src"
    cat = strip_comments((src / "lifted-wavelets.hpp").read_text())
    common = (src / "lifted-common.hpp").read_text()
    wav_block = common[common.index("#define LIFTED_WAVELETS"):]
    wav_block = wav_block[: wav_block.index("#endif")]
    enum = [(m.group(1), int(m.group(2))) for m in ENUM_RE.finditer(wav_block)]

    classes = {m.group(1): m.group(2) for m in CLASS_RE.finditer(cat)}
    rows = []
    wavelets = []
    max_taps = 1
    for name, value in enum:
        body = classes[name]
        defs = {}
        for m in STEP_RE.finditer(body):
            var, fn, targs, args = m.groups()
            defs[var] = (fn, targs, split_args(args))
        order_m = re.search(r"steps\s*=\s*std::make_tuple\((.*?)\)\s*;", body, re.S)
        order = split_args(order_m.group(1)) if order_m else []
        width = int(re.search(r"width\s*=\s*(\d+)\s*;", body).group(1))
        first = len(rows)
        for var in order:
            fn, targs, args = defs[var]
            if fn == "ScaleStep":
                coefs = args
                rows.append(("LW_K_SCALE", "0", "0", str(len(coefs)), "0", coefs,
                             f"{name}.{var}"))
                continue
            target = "LW_EVENS" if fn.endswith("_s") else "LW_ODDS"
            offset = args[0]
            if fn.startswith("unit_"):
                op = "LW_PM_SUB" if "sub" in targs else "LW_PM_ADD"
                rows.append(("LW_K_UNIT", target, offset, "1", op, [], f"{name}.{var}"))
            elif fn.startswith("repeat_"):
                ntap = targs.strip()
                rows.append(("LW_K_REPEAT", target, offset, ntap, "0", args[1:2],
                             f"{name}.{var}"))
            else:
                coefs = args[1:]
                max_taps = max(max_taps, len(coefs))
                rows.append(("LW_K_GEN", target, offset, str(len(coefs)), "0", coefs,
                             f"{name}.{var}"))
        wavelets.append((name, value, width, first, len(rows) - first))

    out = []
    out.append("/* Generated by gen_catalogue.py from the reference's "
               "src/lifted-wavelets.hpp\n * (jcapriot/lifted).  Do not edit. "
               "One row per lifting step, in the order the\n * reference's "
               "steps tuple lists them.  Coefficient literals are verbatim. */")
    out.append(f"#define LW_CATALOGUE_MAX_TAPS {max_taps}")
    out.append(f"#define LW_CATALOGUE_N_WAVELETS {len(wavelets)}")
    out.append(f"#define LW_CATALOGUE_N_STEPS {len(rows)}")
    out.append("#ifdef LW_CATALOGUE_STEPS")
    out.append("/* kind, target, offset, ntaps, unit_pm, {coefficients} */")
    for kind, target, offset, n, pm, coefs, tag in rows:
        c = ", ".join(coefs) if coefs else "0"
        out.append(f"  {{{kind}, {target}, {offset}, {n}, {pm}, {{{c}}}}}, /* {tag} */")
    out.append("#endif")
    out.append("#ifdef LW_CATALOGUE_SHAPES")
    out.append("/* structure only (usable in constexpr device code): kind, target, "
               "offset, ntaps, unit_pm */")
    for kind, target, offset, n, pm, coefs, tag in rows:
        out.append(f"  {{{kind}, {target}, {offset}, {n}, {pm}}}, /* {tag} */")
    out.append("#endif")
    out.append("#ifdef LW_CATALOGUE_RANGES")
    out.append("/* first step row, step count, width -- in catalogue order */")
    for name, value, width, first, count in wavelets:
        out.append(f"  {{{first}, {count}, {width}}}, /* {name} = {value} */")
    out.append("#endif")
    out.append("#ifdef LW_CATALOGUE_WAVELETS")
    out.append("/* name, enum value, width, first step row, step count */")
    for name, value, width, first, count in wavelets:
        out.append(f'  {{"{name}", {value}u, {width}u, {first}u, {count}u}},')
    out.append("#endif")
    sys.stdout.write("\n".join(out) + "\n")


if __name__ == "__main__":
    main()
