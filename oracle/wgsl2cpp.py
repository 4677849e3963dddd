#!/usr/bin/env python3
"""wgsl2cpp.py — rewrite the reference's WGSL compute shaders as C++ source.

TEST INFRASTRUCTURE ONLY: the output is the reference pin built into
oracle/_ref (git-ignored), never shipped and never committed.

Reads the reference's shaders.js (and config.js for MAX_WALLS / WG_SIZE),
pulls out the WGSL template strings (the WGSL_COMMON prelude and each exported
compute shader), fills the ${...} template slots exactly as the JS module
would on a desktop browser, and rewrites WGSL *syntax* into C++ syntax:

  let x = e;            ->  const auto x = e;
  var x: T = e; / var x: T;  ->  T x = e; / T x{};
  fn f(a: T) -> R {     ->  static inline R f(T a) {
  struct S { a: T, }    ->  struct S { T a; };
  @group @binding var<storage|uniform> b : T   ->  a namespace-scope binding
  1.5 (abstract float)  ->  1.5f;  v.xyz -> v.xyz();  i32(e) -> to_i32(e) ...

Expressions are copied token for token, so every arithmetic operation and its
association stays the reference's.  wgsl_compat.hpp provides the builtins.
Each shader lands in its own namespace (wgsl_rt::WGSL_<NAME>) because every
shader re-declares the prelude and its own bindings.
"""
import argparse
import re
import sys


def split_top(s, sep=","):
    """Split on `sep` at bracket depth 0 (<> () [])."""
    out, depth, cur = [], 0, []
    for ch in s:
        if ch in "<([":
            depth += 1
        elif ch in ">)]":
            depth -= 1
        if ch == sep and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(ch)
    out.append("".join(cur))
    return [x.strip() for x in out if x.strip()]


def strip_comments(src):
    return re.sub(r"//[^\n]*", "", src)


FLOAT_RE = re.compile(r"(?<![\w.])(\d+\.\d*(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


class Translator:
    def __init__(self):
        self.fields = set()

    def struct(self, m):
        name, body = m.group(1), m.group(2)
        decls = []
        for f in split_top(body):
            fname, ftype = [x.strip() for x in f.split(":", 1)]
            self.fields.add(fname)
            decls.append(f"    {self.type(ftype)} {fname};")
        return f"struct {name} {{\n" + "\n".join(decls) + "\n};\n"

    @staticmethod
    def type(t):
        t = t.strip()
        m = re.fullmatch(r"array<(.+),\s*(\d+)>", t)
        if m:
            return f"array<{Translator.type(m.group(1))}, {m.group(2)}>"
        return t

    def binding(self, m):
        space, name, ty = m.group(1), m.group(2), m.group(3).strip()
        if space.startswith("uniform"):
            return f"static {ty} {name};"
        am = re.fullmatch(r"array<(.+)>", ty)
        if am and "," not in split_top(am.group(1))[0] and len(split_top(am.group(1))) == 1:
            return f"static {am.group(1)}* {name} = nullptr;"
        return f"static {ty} {name};"

    def func(self, m):
        name, params, ret = m.group(1), m.group(2), m.group(4)
        ps = []
        for p in split_top(params):
            pn, pt = [x.strip() for x in p.split(":", 1)]
            ps.append(f"{pt} {pn}")
        r = ret.strip() if ret else "void"
        return f"static inline {r} {name}({', '.join(ps)}) {{"

    def translate(self, src):
        s = strip_comments(src)
        s = re.sub(r"@compute\s*@workgroup_size\([^)]*\)\s*", "", s)
        s = re.sub(r"@builtin\(\w+\)\s*", "", s)
        s = re.sub(r"struct\s+(\w+)\s*\{(.*?)\}\s*;?", self.struct, s, flags=re.S)
        s = re.sub(r"@group\(\d+\)\s*@binding\(\d+\)\s*var<([^>]*)>\s*(\w+)\s*:\s*([^;]+);",
                   self.binding, s)
        s = re.sub(r"\bfn\s+(\w+)\s*\(([^)]*)\)\s*(->\s*([^{]+?))?\s*\{", self.func, s)
        # module-scope constants
        s = re.sub(r"\bconst\s+(\w+)\s*:\s*([\w<>]+)\s*=", r"static const \2 \1 =", s)
        # declarations
        s = re.sub(r"\blet\s+(\w+)\s*:\s*([^=;]+?)\s*=", r"const \2 \1 =", s)
        s = re.sub(r"\blet\s+(\w+)\s*=", r"const auto \1 =", s)
        s = re.sub(r"\bvar\s+(\w+)\s*:\s*([^=;]+?)\s*=", r"\2 \1 =", s)
        s = re.sub(r"\bvar\s+(\w+)\s*:\s*([^=;]+?)\s*;", lambda m: f"{self.type(m.group(2))} {m.group(1)}{{}};", s)
        s = re.sub(r"\bvar\s+(\w+)\s*=", r"auto \1 =", s)
        # value constructors / conversions of scalars
        s = re.sub(r"(?<![<\w])(i32|u32|f32)\(", r"to_\1(", s)
        # abstract-float literals become f32 literals
        s = FLOAT_RE.sub(lambda m: m.group(1) + "f", s)
        # multi-component swizzles (struct members with such names excluded)
        def swz(m):
            nm = m.group(1)
            if nm in self.fields:
                return m.group(0)
            return f".{nm}()"
        s = re.sub(r"\.([xyzw]{2,4})\b(?!\s*\()", swz, s)
        # WGSL allows a trailing comma in an argument list; C++ does not
        s = re.sub(r",(\s*)\)", r"\1)", s)
        return s


def extract(shaders_js, config_js):
    src = open(shaders_js, encoding="utf-8").read()
    cfg = open(config_js, encoding="utf-8").read()
    max_walls = re.search(r"MAX_WALLS\s*=\s*(\d+)", cfg).group(1)
    wg = re.search(r"WG_SIZE\s*=\s*isMobile\s*\?\s*(\d+)\s*:\s*(\d+)", cfg).group(2)
    band = float(re.search(r"const FLOOR_SPRING_BAND\s*=\s*([0-9.]+)", src).group(1))

    def fill(t):
        t = t.replace("${WG_SIZE}", wg).replace("${MAX_WALLS}", max_walls)
        t = t.replace("${FLOOR_SPRING_BAND.toFixed(1)}", f"{band:.1f}")
        if "${" in t:
            raise SystemExit("unhandled template slot: " + t[t.index("${"):][:60])
        return t

    common = fill(re.search(r"const WGSL_COMMON = /\* wgsl \*/`(.*?)`;", src, re.S).group(1))
    shaders = []
    for m in re.finditer(r"export const (WGSL_\w+) = WGSL_COMMON \+ /\* wgsl \*/`(.*?)`;", src, re.S):
        shaders.append((m.group(1), fill(m.group(2))))
    return common, shaders


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--shaders", required=True)
    ap.add_argument("--config", required=True)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    common, shaders = extract(a.shaders, a.config)
    out = ["// Generated by oracle/wgsl2cpp.py from the reference's shaders.js.",
           "// Test infrastructure (reference pin); not committed.",
           "#pragma once", '#include "../wgsl_compat.hpp"', "namespace wgsl_rt {"]
    for name, body in shaders:
        t = Translator()
        code = t.translate(common + "\n" + body)
        out.append(f"namespace {name} {{\n{code}\n}}  // namespace {name}\n")
    out.append("}  // namespace wgsl_rt\n")
    open(a.out, "w", encoding="utf-8").write("\n".join(out))
    print(f"wgsl2cpp: {len(shaders)} shaders -> {a.out}", file=sys.stderr)


if __name__ == "__main__":
    main()
