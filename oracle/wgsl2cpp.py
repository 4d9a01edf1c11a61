"""ORACLE BUILD STEP — test infrastructure, not product code.

Mechanical translation of the reference's WGSL gas kernels to C++, so that the
reference's own shader text runs here on the CPU (no WebGPU exists on this
machine). Reads, from the reference checkout:

  shaders/{common,advect,diffuse,sources,forces,pressure,geometry,radiation}.wgsl
  js/gpu.js   (genSampler's template literals, taken verbatim; loadWGSL's
               //#include and //#sampler expansion is restated here)

and writes one C++ header with a namespace per shader. The translation is
token by token: WGSL types map to the runtime types of wgsl_rt.hpp, literals
keep WGSL's abstract-float semantics (exact until they meet an f32),
`let`/`var` concretise like WGSL, struct constructors become aggregates. No
expression of the shaders is rewritten by hand.

    python oracle/wgsl2cpp.py <reference root> <out header>
"""
from __future__ import annotations

import os
import re
import sys

SHADERS = ["advect", "diffuse", "sources", "forces", "pressure", "geometry", "radiation", "render"]
TYPE_MAP = {"f32": "float", "i32": "int32_t", "u32": "uint32_t", "bool": "bool",
            "vec2f": "vec2f", "vec3f": "vec3f", "vec3u": "vec3u", "vec4f": "vec4f", "vec2i": "vec2i"}
CPP_RESERVED = {"main": "main_", "near": "near_", "far": "far_", "union": "union_", "char": "char_"}


# ----------------------------------------------------------------------------- js/gpu.js samplers
def sampler_templates(gpu_js: str):
    """The template literals of genSampler in source order, and its ty/off string literals."""
    start = gpu_js.index("function genSampler")
    depth, k = 0, gpu_js.index("{", start)
    end = k
    while True:
        c = gpu_js[end]
        if c == "`":   # skip template literal (may contain braces)
            end = gpu_js.index("`", end + 1)
        elif c == "{":
            depth += 1
        elif c == "}":
            depth -= 1
            if depth == 0:
                break
        end += 1
    body = gpu_js[start:end + 1]
    tpl = re.findall(r"`(.*?)`", body, re.S)
    ty = re.search(r"const ty = kind === 'C' \? '([^']+)' : '([^']+)'", body).groups()
    off = re.search(r"const off = kind === 'U' \? '([^']+)' : '([^']+)'", body).groups()
    if len(tpl) != 6:
        raise RuntimeError(f"genSampler: expected 6 template literals, found {len(tpl)}")
    return tpl, ty, off


def gen_sampler(kind, name, amb, tpl, ty, off):
    """genSampler(kind, name, amb) of js/gpu.js: select the literal and fill its ${...} slots."""
    mm_c, mm_c4, ret_c, fetch_u, fetch_v, ret_uv = tpl

    def fill(s, env):
        return re.sub(r"\$\{(\w+)\}", lambda m: env[m.group(1)], s)

    if kind in ("C", "C4"):
        env = {"name": name, "amb": amb, "ty": ty[0] if kind == "C" else ty[1]}
        env["mm"] = fill(mm_c if kind == "C" else mm_c4, env)
        return fill(ret_c, env)
    if kind in ("U", "V"):
        env = {"name": name}
        env["fetch"] = fill(fetch_u if kind == "U" else fetch_v, env)
        env["off"] = off[0] if kind == "U" else off[1]
        return fill(ret_uv, env)
    raise RuntimeError("unknown sampler kind " + kind)


def load_wgsl(root, name, tpl, ty, off):
    """loadWGSL (js/gpu.js): expand //#include and //#sampler lines."""
    out = []
    for line in open(os.path.join(root, "shaders", name + ".wgsl")).read().splitlines():
        m = re.match(r"^\s*//#include\s+(\w+)", line)
        s = re.match(r"^\s*//#sampler\s+(\w+)\s+(\w+)\s*(.*)$", line)
        if m:
            out.append(open(os.path.join(root, "shaders", m.group(1) + ".wgsl")).read())
        elif s:
            out.append(gen_sampler(s.group(1), s.group(2), s.group(3).strip(), tpl, ty, off))
        else:
            out.append(line)
    return "\n".join(out)


# ----------------------------------------------------------------------------- tokens
TOKEN = re.compile(r"""
    (?P<comment>//[^\n]*)
  | (?P<ws>\s+)
  | (?P<num>0x[0-9a-fA-F]+[ui]?|(?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?f?|\d+[eE][-+]?\d+f?|\d+[uif]?)
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op>->|<<|>>|<=|>=|==|!=|&&|\|\||\+\+|--|\+=|-=|\*=|/=|&=|\|=|[-+*/%&|^!~<>=(){}\[\],;:.@])
""", re.X)


def tokenize(src):
    toks, pos = [], 0
    while pos < len(src):
        m = TOKEN.match(src, pos)
        if not m:
            raise RuntimeError(f"cannot tokenize at: {src[pos:pos + 40]!r}")
        kind = m.lastgroup
        if kind not in ("ws", "comment"):
            toks.append((kind, m.group()))
        pos = m.end()
    return toks


def num_lit(s):
    if s.startswith("0x"):
        return s if s.endswith("u") else s.rstrip("i")
    if s.endswith("u"):
        return s
    if s.endswith("i"):
        return s[:-1]
    if s.endswith("f"):
        return f"float({s[:-1]})"
    if "." in s or "e" in s or "E" in s:
        return f"AF({s})"
    return s   # abstract int: a C++ int


class Translator:
    def __init__(self, toks, ns):
        self.t, self.i, self.ns = toks, 0, ns
        self.structs, self.bindings, self.entries = set(), [], []
        # C++ needs declarations first: structs, then module-scope constants and
        # variables, then prototypes, then function bodies (WGSL allows any order)
        self.s_out, self.v_out, self.protos, self.out = [], [], [], []
        self.uses_barrier = {}

    def peek(self, k=0):
        j = self.i + k
        return self.t[j] if j < len(self.t) else ("eof", "")

    def take(self, val=None):
        tok = self.t[self.i]
        if val is not None and tok[1] != val:
            raise RuntimeError(f"expected {val!r}, found {tok[1]!r} near token {self.i}")
        self.i += 1
        return tok[1]

    # types: f32, vec2f, array<T>, array<T, N>, atomic<i32>, MM4 ...
    def parse_type(self):
        name = self.take()
        if name in ("array", "atomic"):
            self.take("<")
            inner = self.parse_type()
            n = None
            if self.peek()[1] == ",":
                self.take(",")
                n = self.take()
            if self.peek()[1] == ">>":   # array<atomic<i32>>: the outer '>' is left for the caller
                self.t[self.i] = ("op", ">")
            else:
                self.take(">")
            return (name, inner, n)
        return TYPE_MAP.get(name, name)

    def ctype(self, ty):
        if isinstance(ty, tuple):
            kind, inner, n = ty
            if kind == "atomic":
                return self.ctype(inner)
            return f"{self.ctype(inner)}*" if n is None else (self.ctype(inner), n)
        return ty

    # ---- expressions: copy tokens, fixing literals, bitcast<>, struct constructors, builtins casts
    def expr_until(self, stops):
        parts, depth = [], 0
        while True:
            kind, v = self.peek()
            if depth == 0 and v in stops:
                break
            if kind == "eof":
                raise RuntimeError("unexpected end of input in expression")
            if v in "([":
                depth += 1
            elif v in ")]":
                depth -= 1
            self.i += 1
            if kind == "num":
                parts.append(num_lit(v))
            elif kind == "id" and v == "bitcast":
                self.take("<")
                ty = self.parse_type()
                self.take(">")
                parts.append(f"bitcast_{ty}")
            elif kind == "id" and v in self.structs and self.peek()[1] == "(":
                # struct constructor -> aggregate
                self.take("(")
                args = self.expr_until({")"})
                self.take(")")
                parts.append(f"{v}{{{args}}}")
            elif kind == "id" and v in ("f32", "i32", "u32") and self.peek()[1] == "(":
                parts.append({"f32": "conv_f32", "i32": "conv_i32", "u32": "conv_u32"}[v])
            elif kind == "id" and v == "array" and self.peek()[1] == "<":
                raise RuntimeError("array constructors are not used by the gas kernels")
            elif kind == "id":
                parts.append(CPP_RESERVED.get(v, TYPE_MAP.get(v, v)))
            else:
                parts.append(v)
        return " ".join(parts)

    def block(self, indent, fname):
        self.take("{")
        lines = []
        while self.peek()[1] != "}":
            lines.extend(self.statement(indent + "  ", fname))
        self.take("}")
        return lines

    def statement(self, ind, fname):
        kind, v = self.peek()
        if v in ("let", "var", "const"):
            self.take()
            name = self.take()
            ty = None
            if self.peek()[1] == ":":
                self.take(":")
                ty = self.parse_type()
            init = None
            if self.peek()[1] == "=":
                self.take("=")
                init = self.expr_until({";"})
            self.take(";")
            name = CPP_RESERVED.get(name, name)
            if ty is not None:
                ct = self.ctype(ty)
                return [f"{ind}{'const ' if v != 'var' else ''}{ct} {name} = conv<{ct}>({init});" if init
                        else f"{ind}{ct} {name}{{}};"]
            q = "const auto" if v != "var" else "auto"
            return [f"{ind}{q} {name} = conc({init});"]
        if v == "if":
            self.take()
            self.take("(")
            cond = self.expr_until({")"})
            self.take(")")
            lines = [f"{ind}if ({cond}) {{"] + self.block(ind, fname) + [f"{ind}}}"]
            while self.peek()[1] == "else":
                self.take()
                if self.peek()[1] == "if":
                    self.take()
                    self.take("(")
                    c2 = self.expr_until({")"})
                    self.take(")")
                    lines += [f"{ind}else if ({c2}) {{"] + self.block(ind, fname) + [f"{ind}}}"]
                else:
                    lines += [f"{ind}else {{"] + self.block(ind, fname) + [f"{ind}}}"]
            return lines
        if v == "for":
            self.take()
            self.take("(")
            init = self.statement("", fname)[0].strip().rstrip(";")
            cond = self.expr_until({";"})
            self.take(";")
            step = self.expr_until({")"})
            self.take(")")
            return [f"{ind}for ({init}; {cond}; {step}) {{"] + self.block(ind, fname) + [f"{ind}}}"]
        if v in ("return", "continue", "break"):
            self.take()
            e = self.expr_until({";"})
            self.take(";")
            return [f"{ind}{v} {e};".replace(" ;", ";")]
        if v == "{":
            return [f"{ind}{{"] + self.block(ind, fname) + [f"{ind}}}"]
        e = self.expr_until({";"})
        self.take(";")
        if "workgroupBarrier" in e:
            self.uses_barrier[fname] = True
        return [f"{ind}{e};"]

    def top(self):
        attrs = []
        while self.peek()[0] != "eof":
            kind, v = self.peek()
            if v == "@":
                self.take()
                a = self.take()
                args = ""
                if self.peek()[1] == "(":
                    self.take("(")
                    args = self.expr_until({")"})
                    self.take(")")
                attrs.append((a, args))
                continue
            if v == "struct":
                self.take()
                name = self.take()
                self.structs.add(name)
                self.take("{")
                fields = []
                while self.peek()[1] != "}":
                    while self.peek()[1] == "@":   # @builtin(position), @location(n): interface attributes
                        self.take("@")
                        self.take()
                        if self.peek()[1] == "(":
                            self.take("(")
                            self.expr_until({")"})
                            self.take(")")
                    fname = CPP_RESERVED.get(self.take(), None) or self.t[self.i - 1][1]
                    self.take(":")
                    fty = self.ctype(self.parse_type())
                    fields.append(f"  {fty} {fname};")
                    if self.peek()[1] == ",":
                        self.take(",")
                self.take("}")
                if self.peek()[1] == ";":
                    self.take(";")
                self.s_out += [f"struct {name} {{"] + fields + ["};"]
                attrs = []
                continue
            if v == "const":
                self.v_out.append("static " + self.statement("", "")[0])
                attrs = []
                continue
            if v == "var":
                self.take()
                space = None
                if self.peek()[1] == "<":
                    self.take("<")
                    space = self.expr_until({">"})
                    self.take(">")
                name = self.take()
                self.take(":")
                ty = self.parse_type()
                self.take(";")
                group = [a for a in attrs if a[0] == "binding"]
                if space and space.startswith("workgroup"):
                    et, n = self.ctype(ty)
                    self.v_out.append(f"static {et} {name}[{n}];")
                elif space and space.startswith("uniform"):
                    self.v_out.append(f"static {self.ctype(ty)} {name};")
                    self.bindings.append((name, "uniform", self.ctype(ty)))
                else:
                    self.v_out.append(f"static {self.ctype(ty)} {name} = nullptr;")
                    self.bindings.append((name, "storage", self.ctype(ty)))
                attrs = []
                continue
            if v == "fn":
                self.take()
                name = self.take()
                self.take("(")
                params, builtins = [], []
                while self.peek()[1] != ")":
                    battr = None
                    if self.peek()[1] == "@":
                        self.take("@")
                        self.take("builtin")
                        self.take("(")
                        battr = self.take()
                        self.take(")")
                    pname = self.take()
                    self.take(":")
                    pty = self.ctype(self.parse_type())
                    params.append(f"{pty} {CPP_RESERVED.get(pname, pname)}")
                    builtins.append(battr)
                    if self.peek()[1] == ",":
                        self.take(",")
                self.take(")")
                ret = "void"
                if self.peek()[1] == "->":
                    self.take("->")
                    while self.peek()[1] == "@":   # -> @location(0) vec4f
                        self.take("@")
                        self.take()
                        self.take("(")
                        self.expr_until({")"})
                        self.take(")")
                    ret = self.ctype(self.parse_type())
                cname = CPP_RESERVED.get(name, name)
                if any(a[0] == "vertex" for a in attrs):
                    # the full-screen triangle's vertex stage: the harness computes the
                    # fragment's interpolated position itself, so the body is not needed
                    depth = 0
                    while True:
                        v2 = self.take()
                        depth += v2 == "{"
                        depth -= v2 == "}"
                        if depth == 0 and v2 == "}":
                            break
                    attrs = []
                    continue
                body = self.block("", cname)
                self.protos.append(f"static {ret} {cname}({', '.join(params)});")
                self.out += [f"static {ret} {cname}({', '.join(params)}) {{"] + body + ["}"]
                ws = [a for a in attrs if a[0] == "workgroup_size"]
                if ws:
                    dims = [int(x) for x in ws[0][1].replace(" ", "").split(",")]
                    while len(dims) < 3:
                        dims.append(1)
                    self.entries.append((cname, dims, builtins))
                attrs = []
                continue
            raise RuntimeError(f"unexpected top-level token {v!r}")

    def emit(self):
        L = ([f"namespace {self.ns} {{", "using namespace wgsl;"] + self.s_out + self.v_out + self.protos
             + self.out)
        # bind(name, pointer): the bind group of a dispatch (js/gpu.js Kernel.bind)
        L.append("static void bind(const char* name, void* ptr) {")
        for name, kind, ct in self.bindings:
            if kind == "uniform":
                L.append(f"  if (!std::strcmp(name, \"{name}\")) {{ std::memcpy(&{name}, ptr, sizeof {name}); return; }}")
            else:
                L.append(f"  if (!std::strcmp(name, \"{name}\")) {{ {name} = reinterpret_cast<{ct}>(ptr); return; }}")
        L.append("}")
        for name, dims, builtins in self.entries:
            args = []
            for b in builtins:
                args.append({"global_invocation_id": "gid", "workgroup_id": "wgid",
                             "local_invocation_index": "li", "local_invocation_id": "lid"}[b])
            call = f"{name}({', '.join(args)})"
            barrier = "true" if self.uses_barrier.get(name) else "false"
            L.append(f"static void dispatch_{name}(uint32_t wx, uint32_t wy, uint32_t wz) {{")
            L.append(f"  wgsl::dispatch({dims[0]}, {dims[1]}, {dims[2]}, wx, wy, wz, {barrier},")
            L.append(f"      [](vec3u gid, vec3u wgid, vec3u lid, uint32_t li) {{ (void)gid; (void)wgid; (void)lid; (void)li; {call}; }});")
            L.append("}")
        L.append(f"}}  // namespace {self.ns}")
        return "\n".join(L)


def main(root, out_path):
    gpu_js = open(os.path.join(root, "js", "gpu.js")).read()
    tpl, ty, off = sampler_templates(gpu_js)
    parts = ["// Generated by oracle/wgsl2cpp.py from the reference's shaders/*.wgsl and js/gpu.js.",
             "// Test infrastructure: do not edit, regenerate.", "#pragma once", '#include "wgsl_rt.hpp"']
    for s in SHADERS:
        src = load_wgsl(root, s, tpl, ty, off)
        tr = Translator(tokenize(src), f"wgsl_{s}")
        tr.top()
        parts.append(tr.emit())
    os.makedirs(os.path.dirname(os.path.abspath(out_path)), exist_ok=True)
    open(out_path, "w").write("\n\n".join(parts) + "\n")


if __name__ == "__main__":
    main(sys.argv[1], sys.argv[2])
