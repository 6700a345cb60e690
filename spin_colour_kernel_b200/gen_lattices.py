"""Generate csrc/lattices.h: compile-time bond tables of the common crystals.

    python -m spin_colour_kernel_b200.gen_lattices

For each (crystal, shells) below, the bond list of every sublattice in local-field accumulation order for
distinct non-zero couplings per shell (one coupling group per shell, shells ascending, bonds in table order)
becomes a constexpr table. A system whose lowered descriptor equals one of these tables runs the specialised
class kernels, where every neighbour offset is a compile-time constant; any other system runs the generic
kernels. The tables come from crystals.make, so they follow the reference's bond order.
"""

from __future__ import annotations

from pathlib import Path

from .crystals import make

SPECS = [
    ("square", (1,)),
    ("triangular", (1,)),
    ("sc", (1,)),
    ("bcc", (1,)),
    ("bcc", (1, 2)),
    ("fcc", (1,)),
]

OUT = Path(__file__).resolve().parent / "csrc" / "lattices.h"


def spec_name(crystal: str, shells) -> str:
    return f"Lat_{crystal}_{'_'.join(map(str, shells))}"


def render() -> str:
    lines = [
        "// GENERATED by spin_colour_kernel_b200/gen_lattices.py from crystals.make: do not edit by hand.",
        "// Compile-time bond tables (one coupling group per shell) of the specialised class kernels.",
        "#pragma once",
        "",
        "#include <stdint.h>",
        "",
        "namespace sck {",
        "",
        "struct BondC {",
        "  int a2, dx, dy, dz;",
        "};",
        "",
    ]
    ids = []
    for sid, (name, shells) in enumerate(SPECS):
        c = make(name, shells)
        per_alpha = []
        for a in range(c.b):
            bonds = [bd for s in sorted(shells) for bd in c.bonds if bd.alpha == a and bd.shell == s]
            ends, n = [], 0
            for s in sorted(shells):
                n += sum(1 for bd in c.bonds if bd.alpha == a and bd.shell == s)
                ends.append(n)
            per_alpha.append((bonds, ends))
        reach = max(abs(v) for bd in c.bonds for v in bd.delta)
        nmax = max(len(b) for b, _ in per_alpha)
        sname = spec_name(name, shells)
        ids.append(sname)
        lines.append(f"// {name}, shells {tuple(shells)}: b = {c.b}, D = {c.D}, reach {reach}")
        lines.append(f"struct {sname} {{")
        lines.append(f"  static constexpr int id = {sid + 1};")
        lines.append(f"  static constexpr int b = {c.b};")
        lines.append(f"  static constexpr int dim = {c.D};")
        lines.append(f"  static constexpr int reach = {reach};")
        lines.append(f"  static constexpr int groups = {len(shells)};")
        lines.append(f"  static constexpr int max_bonds = {nmax};")
        counts = ", ".join(str(len(b)) for b, _ in per_alpha)
        lines.append(f"  __host__ __device__ static constexpr int n_bonds(int a) {{")
        lines.append(f"    constexpr int t[{c.b}] = {{{counts}}};")
        lines.append("    return t[a];")
        lines.append("  }")
        ends = ", ".join("{" + ", ".join(map(str, e)) + "}" for _, e in per_alpha)
        lines.append("  __host__ __device__ static constexpr int group_end(int a, int g) {")
        lines.append(f"    constexpr int t[{c.b}][{len(shells)}] = {{{ends}}};")
        lines.append("    return t[a][g];")
        lines.append("  }")
        rows = []
        for bonds, _ in per_alpha:
            padded = [(bd.alpha2, *(list(bd.delta) + [0] * (3 - c.D))) for bd in bonds]
            padded += [(0, 0, 0, 0)] * (nmax - len(bonds))
            rows.append("{" + ", ".join("{%d, %d, %d, %d}" % t for t in padded) + "}")
        lines.append("  __host__ __device__ static constexpr BondC bond(int a, int i) {")
        lines.append(f"    constexpr BondC t[{c.b}][{nmax}] = {{")
        for r in rows:
            lines.append(f"        {r},")
        lines.append("    };")
        lines.append("    return t[a][i];")
        lines.append("  }")
        lines.append("};")
        lines.append("")
    lines.append(f"constexpr int kLatticeSpecs = {len(SPECS)};")
    lines.append("")
    lines.append("}  // namespace sck")
    lines.append("")
    return "\n".join(lines)


def main():
    OUT.write_text(render())
    print(OUT)


if __name__ == "__main__":
    main()
