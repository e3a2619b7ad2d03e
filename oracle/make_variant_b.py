"""Write the bug-fixed ("variant B") copies of two reference files for the
CPU oracle build. Test infrastructure: the copies go to oracle/_ref/src_B/,
which is git-ignored and only ever compiled into oracle/_ref/libref_B.so.

The three fixes, each a one-line change of an evident slip:
  OST/ost.ver2.c:75    q5 (Qyz) accumulates m*dy*dx; fixed to m*dy*dz.
  OST/ost.ver2.c:273-275  AddNode adds the x component three times to
                       axyz[0]; fixed to add x, y, z to axyz[0], [1], [2].
  Cosmos/treecorrection.c:214-216  DirectSummation adds every target's force
                       to pos->axyz (the first target); fixed to pos[i].axyz.

Usage: python make_variant_b.py <reference_root> <out_dir>
"""
import os
import sys


def patch(text, old, new, count):
    n = text.count(old)
    if n != count:
        raise SystemExit(f"variant B patch: expected {count} match(es) of {old!r}, found {n}")
    return text.replace(old, new)


def main():
    ref, out = sys.argv[1], sys.argv[2]
    os.makedirs(out, exist_ok=True)
    ost = open(os.path.join(ref, "OST", "ost.ver2.c")).read()
    ost = patch(ost, "q5 += ptlmass * tmpy*tmpx;", "q5 += ptlmass * tmpy*tmpz;", 1)
    line = "(p->axyz[0]) += vfact2*(tmpx*tmptmp + qxx1 * twofplmf2);"
    fixed = ("(p->axyz[0]) += vfact2*(tmpx*tmptmp + qxx1 * twofplmf2);\\\n"
             "\t\t(p->axyz[1]) += vfact2*(tmpy*tmptmp + qxx2 * twofplmf2);\\\n"
             "\t\t(p->axyz[2]) += vfact2*(tmpz*tmptmp + qxx3 * twofplmf2);")
    block_old = (line + "\\\n\t\t" + line + "\\\n\t\t" + line)
    ost = patch(ost, block_old, fixed, 1)
    open(os.path.join(out, "ost.ver2.c"), "w").write(ost)

    tc = open(os.path.join(ref, "Cosmos", "treecorrection.c")).read()
    for c, v in (("0", "ax"), ("1", "ay"), ("2", "az")):
        tc = patch(tc, f"\t\tpos->axyz[{c}] += vfact2*{v};", f"\t\tpos[i].axyz[{c}] += vfact2*{v};", 1)
    open(os.path.join(out, "treecorrection.c"), "w").write(tc)


if __name__ == "__main__":
    main()
