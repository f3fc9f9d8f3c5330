"""Build-time overlay for compiling the apxchol reference with g++ 13.

g++ 13 lacks C++23 "deducing this", which two reference headers use:
  include/apxchol/checkpoint.h:73          (recursive lambda in report())
  include/apxchol/graph/forward_star.h:325 (operator[] on const/non-const self)
This script copies those two headers from the reference tree into an overlay
directory (placed first on the include path) and rewrites only those
constructs into equivalent C++20. The output goes to a git-ignored build
folder; no reference source is committed. Each substitution must match
exactly once, so a changed reference fails loudly instead of compiling
something else.

usage: python patch_ref.py <reference_root> <overlay_dir>
"""
import os
import sys


def _sub_once(text, old, new, where):
    n = text.count(old)
    if n != 1:
        raise SystemExit(f"patch_ref: expected exactly one match in {where}, found {n}: {old!r}")
    return text.replace(old, new)


def main(ref_root, overlay):
    inc = os.path.join(ref_root, "include")
    # checkpoint.h: recursive lambda taking itself explicitly.
    src = os.path.join(inc, "apxchol", "checkpoint.h")
    t = open(src).read()
    t = _sub_once(t, "[&](this auto const& collect, const node& n,",
                  "[&](auto const& collect, const node& n,", src)
    t = _sub_once(t, "collect(c, depth + 1)", "collect(collect, c, depth + 1)", src)
    t = _sub_once(t, "collect(root_, 0)", "collect(collect, root_, 0)", src)
    dst = os.path.join(overlay, "apxchol", "checkpoint.h")
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    open(dst, "w").write(t)

    # forward_star.h: one deducing-this operator[] -> const and non-const overloads.
    src = os.path.join(inc, "apxchol", "graph", "forward_star.h")
    t = open(src).read()
    old = ("    template<typename Self>\n"
           "    auto operator[](this Self&& self, node_index v) {\n"
           "        return std::ranges::subrange(\n"
           "            iterator_<Self>{&self, self.head_[v]}, std::default_sentinel);\n"
           "    }\n")
    new = ("    auto operator[](node_index v) {\n"
           "        return std::ranges::subrange(\n"
           "            iterator_<decltype(*this)>{this, head_[v]}, std::default_sentinel);\n"
           "    }\n"
           "    auto operator[](node_index v) const {\n"
           "        return std::ranges::subrange(\n"
           "            iterator_<decltype(*this)>{this, head_[v]}, std::default_sentinel);\n"
           "    }\n")
    t = _sub_once(t, old, new, src)
    dst = os.path.join(overlay, "apxchol", "graph", "forward_star.h")
    os.makedirs(os.path.dirname(dst), exist_ok=True)
    open(dst, "w").write(t)


if __name__ == "__main__":
    if len(sys.argv) != 3:
        raise SystemExit(__doc__)
    main(sys.argv[1], sys.argv[2])
