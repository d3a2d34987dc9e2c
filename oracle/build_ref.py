"""Build recipe for oracle/_ref: the reference's own code, compiled here.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this file or the
library it builds; tests/, the smoke check and bench.py's CPU-baseline leg use
the result as a checker / reference timing.

What it compiles, from the sources where they lie under the reference tree
(REF_ROOT: MYRT_REFERENCE_ROOT, by default the checkout beside this
repository, ../reference; here /root/reference):

* src/pathtracer/bvh.cpp and src/thread_pool.cpp with the two shims under
  oracle/shim (rnu vector math, <experimental/generator>). bvh.cpp needs one
  build-time edit: the explicit ``myrt::`` qualification on
  ``generate_triangle_bounds`` at bvh.cpp:136 is an MSVC-ism that g++ rejects,
  so a copy with that token removed is written to oracle/_ref/src/.
* The shader helper files src/pt/{random,intersect,ggx,color,pbr,transform,
  bvh,bvh.impl}.glsl and the traversal visitors of src/pt/pt_trace.comp
  (lines 229-309: traversal_state_t, traversal_init, visit_triangle and the
  instance visitor visit_object_aabb; the drawable record of lines 34-47),
  compiled
  as C++ through oracle/glsl_compat.hpp after these mechanical rewrites only:
    - ``out T x`` / ``inout T x`` parameters -> ``T& x``; ``const in`` -> ``const``;
    - float literals without a suffix get ``f`` (GLSL literals are float);
    - per-invocation globals become ``thread_local``.
  The rewritten copies go to oracle/_ref/glsl/.
* The post-processing shaders src/pt/pp_*.comp (ref_harness_post.cpp), the
  forward renderer's resolve pass src/pt/forward/resolve.frag and the path
  tracer's generate and color passes src/pt/pt_generate.comp,
  src/pt/pt_color.comp with src/pt/bokeh.glsl (ref_harness_glsl.cpp, see
  resolve_to_cpp and pass_to_cpp), with the rewrites their converters list.

Output: oracle/_ref/libmyrt_ref.so (git-ignored; it travels with the tree).
The reference tree is only needed at build time.
"""
from __future__ import annotations

import os
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
# the reference checkout beside this repository (../reference), or MYRT_REFERENCE_ROOT
REF_ROOT = Path(os.environ.get("MYRT_REFERENCE_ROOT", HERE.parent.parent / "reference")).resolve()

GLSL_FILES = ["random.glsl", "intersect.glsl", "ggx.glsl", "color.glsl", "pbr.glsl", "transform.glsl", "bvh.glsl",
              "bvh.impl.glsl"]

_FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][-+]?\d+)?|\d+[eE][-+]?\d+)(?![\w.])")
_PARAM_REF = re.compile(r"\b(?:inout|out)\s+([A-Za-z_]\w*)\s+([A-Za-z_]\w*)")
_GLOBAL_VAR = re.compile(r"^(int|bool|float|uint|vec3|random_state_t|material_state_t)(\s+\w+\s*(?:=[^;]*)?;)", re.M)


# GLSL evaluates function arguments left to right (GLSL 4.60, 6.1.1); C++ leaves
# the order unspecified and g++ goes right to left. Where one argument list holds
# several draws from the random stream, the draws are hoisted into temporaries in
# source order. Each pattern must match exactly (count given), so a change in the
# reference fails the build instead of silently reordering.
ORDER_FIXES = {
    "random.glsl": [
        (r"int seed_base = int\(random_int\((pixel\.x \^ 0xba77fa)\) \* random_primes\[0\] \+ "
         r"random_int\((pixel\.y \^ 0xcca6df)\) \* random_primes\[1\] \+ random_int\(start_seed\)\);",
         r"int _r0 = random_int(\1); int _r1 = random_int(\2); int _r2 = random_int(start_seed); "
         r"int seed_base = int(_r0 * random_primes[0] + _r1 * random_primes[1] + _r2);", 2),
        (r"return vec2\(random_next\(\), random_next\(\)\);",
         r"float _a = random_next(); float _b = random_next(); return vec2(_a, _b);", 1),
        (r"return vec3\(random_next\(\), random_next\(\), random_next\(\)\);",
         r"float _a = random_next(); float _b = random_next(); float _c = random_next(); return vec3(_a, _b, _c);", 1),
        (r"vec2 rands = vec2\(\s*random_next\(\) \* 2 \* (3\.1415926535897f),\s*random_next\(\)\s*\);",
         r"float _a = random_next() * 2 * \1; float _b = random_next(); vec2 rands = vec2(_a, _b);", 1),
    ],
}


# SDF instruction types of src/pathtracer/sdf.hpp:399-633 whose GLSL snippets
# compile (smooth_subtraction / smooth_intersection use `h` before declaring it
# and compile in no language). Each snippet becomes one C++ function with the
# signature the code generator gives it (sdf.cpp:135-149): prim
# (in_position, inout_material, params...), op (in_distance0/1, in_material0/1,
# inout_material, params...), mod (in_position, out_multiplier, params...).
SDF_TYPES = ["sphere", "translate", "hard_union", "hard_subtraction", "hard_intersection", "smooth_union", "box",
             "torus", "menger_fractal", "vertical_capsule", "mirror_axis"]
_SDF_PARAM_CPP = {"float": "float", "int": "int", "uint": "uint", "vec3": "vec3"}


def extract_sdf_snippets(src: str) -> str:
    out = []
    for name in SDF_TYPES:
        m = re.search(r"struct %s : (prim|op|mod) \{(.*?)\n  \};" % name, src, re.S)
        assert m, f"sdf.hpp: struct {name} not found"
        cat, body = m.group(1), m.group(2)
        g = re.search(r'constexpr static auto glsl = R"\((.*?)\)";', body, re.S)
        if g:
            glsl = g.group(1)
            head = re.search(r"basic_type\{\s*instruction_type::category::\w+,\s*glsl\s*,\s*\{([^}]*)\}", body, re.S)
        else:
            head = re.search(r'basic_type\{\s*instruction_type::category::\w+,\s*(?:R"\((.*?)\)"|"((?:[^"\\]|\\.)*)")'
                             r'\s*,\s*\{([^}]*)\}', body, re.S)
            glsl = head.group(1) if head.group(1) is not None else head.group(2)
        assert head, f"sdf.hpp: basic_type of {name} not found"
        ptypes = re.findall(r"(\w+)_param::type", head.group(head.lastindex))
        params = "".join(f", {_SDF_PARAM_CPP[t]} in_param{i}" for i, t in enumerate(ptypes))
        glsl = glsl.replace("mix_material", "_mxm").replace("load_material", "_ldm")
        if cat == "prim":
            sig = f"float sdf_{name}(vec3 in_position, _MT& inout_material{params})"
        elif cat == "op":
            sig = (f"float sdf_{name}(float in_distance0, float in_distance1, _MT in_material0, _MT in_material1, "
                   f"_MT& inout_material{params})")
        else:
            sig = f"vec3 sdf_{name}(vec3 in_position, float& out_multiplier{params})"
        out.append(f"// sdf.hpp: struct {name} ({cat})\n{sig} {{\n{glsl}\n}}\n")
    return glsl_to_cpp("\n".join(out), globals_thread_local=False)  # snippet bodies hold locals only


def raymarch_to_cpp(src: str) -> str:
    # GLSL lets a float be swizzled (`x.x`); C++ does not. raymarch.glsl:107.
    src, n = re.subn(r"map\(p \+ 0\.0005 \* e / len, dum, true\)\.x", "map(p + 0.0005 * e / len, dum, true)", src)
    assert n == 1, "raymarch.glsl: normal estimate changed"
    return glsl_to_cpp(src)


def fix_evaluation_order(name: str, src: str) -> str:
    for pat, rep, count in ORDER_FIXES.get(name, []):
        src, n = re.subn(pat, rep, src)
        assert n == count, f"{name}: evaluation-order rewrite matched {n} times, expected {count}: {pat}"
    return src


def glsl_to_cpp(src: str, globals_thread_local: bool = True) -> str:
    src = re.sub(r"\bconst\s+in\s+", "const ", src)
    src = re.sub(r"(?<=[(,])\s*in\s+(?=[A-Za-z_]\w*\s+[A-Za-z_]\w*\s*[,)])", " ", src)  # plain `in` parameters
    src = _PARAM_REF.sub(r"\1& \2", src)
    src = _FLOAT_LIT.sub(r"\1f", src)
    if globals_thread_local:
        src = _GLOBAL_VAR.sub(r"thread_local \1\2", src)
    return src


def extract_trace_visitor(src: str) -> str:
    """pt_trace.comp:229-309 (traversal state, traversal_init, visit_triangle and
    the instance visitor visit_object_aabb), up to any_hit()."""
    start = src.index("struct traversal_state_t")
    end = src.index("bool any_hit(vec3 ray_origin, vec3 ray_direction, float max_distance)\n{")
    seg = src[start:end]
    assert "bool visit_object_aabb" in seg, "pt_trace.comp: visit_object_aabb moved"
    seg, n = re.subn(r"\}\s*traversal\s*;", "};\nthread_local traversal_state_t traversal;", seg)
    assert n == 1, "pt_trace.comp: traversal_state_t layout changed"
    return glsl_to_cpp(seg)


def extract_drawable_geometry(src: str) -> str:
    """pt_trace.comp:34-47: the per-drawable record (drawable_geometry_t)."""
    start = src.index("struct drawable_geometry_t")
    end = src.index("};", start) + 2
    return glsl_to_cpp(src[start:end])


def material_codegen(src: str, type_name: str = "material") -> str:
    """The text substitution material_registry::push_type applies (material.hpp:18-29)."""
    for word in ("open", "evaluate", "bounce"):
        src = src.replace(word, f"{type_name}_{word}_")
    src = src.replace("this", f"{type_name}_instance_")
    return f"thread_local {type_name} {type_name}_instance_;\n" + glsl_to_cpp(src)


PP_SHADERS = ["pp_denoise", "pp_blur", "pp_cutoff", "pp_add", "pp_tonemap", "pp_fxaa"]


def pp_to_cpp(name: str, src: str) -> str:
    """A post-processing compute shader as C++ for ref_harness_post.cpp: the
    #version line and the work-group layout go, `layout(...) uniform` /
    `uniform` / `writeonly` qualifiers go (the harness sets the globals), main
    becomes pp_main, swizzles become accessor calls (.rgb(), .xyz(), .xy();
    .a reads .w), and pp_tonemap's one swizzle assignment is spelled out."""
    src = re.sub(r"^#version.*$", "", src, flags=re.M)
    src, n = re.subn(r"^layout\(local_size_x[^)]*\)\s*in\s*;", "", src, flags=re.M)
    assert n == 1, f"{name}: work-group layout not found"
    src = re.sub(r"layout\([^)]*\)\s*uniform\s+", "", src)
    src = re.sub(r"\buniform\s+", "", src)
    src = re.sub(r"\bwriteonly\s+", "", src)
    src, n = re.subn(r"\bvoid\s+main\s*\(\s*\)", "void pp_main()", src)
    assert n == 1, f"{name}: main not found"
    if name == "pp_tonemap":
        src, n = re.subn(r"color\.rgb\s*=\s*tonemap\(color\.rgb\);",
                         "{ vec3 _t = tonemap(color.rgb()); color.x = _t.x; color.y = _t.y; color.z = _t.z; }", src)
        assert n == 1, "pp_tonemap: swizzle assignment changed"
    src = re.sub(r"\.rgb\b(?!\()", ".rgb()", src)
    src = re.sub(r"\.xyz\b(?!\()", ".xyz()", src)
    src = re.sub(r"\.xy\b(?!\()", ".xy()", src)
    src = re.sub(r"\.a\b", ".w", src)
    return glsl_to_cpp(src, globals_thread_local=False)


def resolve_to_cpp(src: str) -> str:
    """src/pt/forward/resolve.frag as C++ for ref_harness_glsl.cpp, which
    includes it inside a namespace of its own after the helper files and the
    material dispatch: the #version / #extension lines and the #include lines
    go (the harness included those files already), interface qualifiers go
    (`layout(...)`, `uniform`, `flat in`, `out` on globals: the harness sets the
    globals per fragment), the two storage buffers become pointers, main
    becomes resolve_main, `uint(x)` of a float becomes to_uint(x) (the
    conversion GLSL leaves undefined for negative values; the harness gives
    NVIDIA's: truncate, saturate, NaN -> 0), and the one swizzle assignment
    `color.rgb = ...` is spelled out per component."""
    src = re.sub(r"^#version.*$", "", src, flags=re.M)
    src = re.sub(r"^#extension.*$", "", src, flags=re.M)
    src, n = re.subn(r'^#include\s+"[^"]*"\s*$', "", src, flags=re.M)
    assert n == 4, f"resolve.frag: expected 4 includes, found {n}"
    src, n = re.subn(r"layout\([^)]*\)\s*restrict\s+readonly\s+buffer\s+\w+\s*\{\s*(\w+)\s+(\w+)\[\]\s*;\s*\}\s*;",
                     r"\1 const* \2 = nullptr;", src)
    assert n == 2, "resolve.frag: storage buffers changed"
    src = re.sub(r"layout\([^)]*\)\s*", "", src)
    src = re.sub(r"^\s*flat\s+in\s+", "", src, flags=re.M)
    src = re.sub(r"^\s*out\s+(?=vec4\s+color\s*;)", "", src, flags=re.M)
    src = re.sub(r"\buniform\s+", "", src)
    src, n = re.subn(r"\bvoid\s+main\s*\(\s*\)", "void resolve_main()", src)
    assert n == 1, "resolve.frag: main not found"
    src, n = re.subn(r"\buint\((?=position\.)", "to_uint(", src)
    assert n == 3, f"resolve.frag: expected 3 uint(position.*) conversions, found {n}"
    src, n = re.subn(r"color\.rgb\s*=\s*background\(ray_direction\);",
                     "{ vec3 _t = background(ray_direction); color.x = _t.x; color.y = _t.y; color.z = _t.z; }", src)
    assert n == 1, "resolve.frag: background assignment changed"
    return glsl_to_cpp(src, globals_thread_local=False)


PASS_SHADERS = {"pt_color": 4, "pt_generate": 3}  # shader -> #include lines it has


def pass_to_cpp(name: str, src: str) -> str:
    """A path-tracer pass (pt_generate.comp, pt_color.comp) as C++ for
    ref_harness_glsl.cpp, which includes it in a namespace of its own after the
    helper files, the material dispatch and the GL stand-ins (images, samplers,
    gl_GlobalInvocationID): the #version / #extension lines, the work-group
    layout, the bindless-sampler default and the #include lines go; a storage
    buffer holding one array becomes a pointer and one holding scalars becomes
    those scalars; interface qualifiers (`layout(...)`, `uniform`) go; main
    becomes pass_main; the unsuffixed literal 2341335623, which GLSL makes an
    int with that bit pattern (GLSL 4.60, 4.1.3), is written as such; the one
    array assignment `result.pad = float[2](0,0);` is spelled out; the two
    random draws in one argument list of pt_color.comp are hoisted in source
    order (GLSL evaluates arguments left to right, C++ leaves it open)."""
    src = re.sub(r"^#version.*$", "", src, flags=re.M)
    src = re.sub(r"^#extension.*$", "", src, flags=re.M)
    src, n = re.subn(r"^layout\(local_size_x[^)]*\)\s*in\s*;", "", src, flags=re.M)
    assert n == 1, f"{name}: work-group layout not found"
    src = re.sub(r"^layout\(bindless_sampler\)\s*uniform\s*;", "", src, flags=re.M)
    src, n = re.subn(r'^#include\s+"[^"]*"\s*$', "", src, flags=re.M)
    assert n == PASS_SHADERS[name], f"{name}: expected {PASS_SHADERS[name]} includes, found {n}"
    src = re.sub(r"layout\([^)]*\)\s*(?:restrict\s+)?(?:readonly\s+|writeonly\s+)?buffer\s+\w+\s*"
                 r"\{\s*(\w+)\s+(\w+)\[\]\s*;\s*\}\s*;", r"\1* \2 = nullptr;", src)
    src = re.sub(r"layout\([^)]*\)\s*(?:restrict\s+)?(?:readonly\s+)?buffer\s+\w+\s*\{([^}]*)\}\s*;", r"\1", src)
    assert "buffer" not in re.sub(r"//.*", "", src), f"{name}: a storage buffer was not rewritten"
    src = re.sub(r"layout\([^)]*\)\s*", "", src)
    src = re.sub(r"\buniform\s+", "", src)
    src, n = re.subn(r"\bvoid\s+main\s*\(\s*\)", "void pass_main()", src)
    assert n == 1, f"{name}: main not found"
    src = src.replace("2341335623", "int(2341335623u)")
    src = src.replace("result.pad = float[2](0,0);", "result.pad[0] = 0; result.pad[1] = 0;")
    if name == "pt_color":
        src, n = re.subn(r"vec2 material_randoms = vec2\(random_next\(\), random_next\(\)\);",
                         "float _r0 = random_next(); float _r1 = random_next(); vec2 material_randoms = vec2(_r0, _r1);",
                         src)
        assert n == 1, "pt_color: material_randoms changed"
    assert not re.search(r"\([^()]*random_\w+\([^()]*\)[^()]*,[^()]*random_\w+\(", src), \
        f"{name}: another argument list with two random draws"
    return glsl_to_cpp(src, globals_thread_local=False)


def write_sources() -> None:
    (OUT / "src").mkdir(parents=True, exist_ok=True)
    (OUT / "glsl").mkdir(parents=True, exist_ok=True)
    bvh_src = (REF_ROOT / "src/pathtracer/bvh.cpp").read_text()
    needle = "std::vector<aabb_t> myrt::generate_triangle_bounds("
    assert bvh_src.count(needle) == 1, "bvh.cpp:136 no longer has the expected qualifier"
    (OUT / "src/bvh.cpp").write_text(bvh_src.replace(needle, "std::vector<aabb_t> generate_triangle_bounds("))
    for name in GLSL_FILES:
        src = glsl_to_cpp((REF_ROOT / "src/pt" / name).read_text())
        (OUT / "glsl" / name).write_text(fix_evaluation_order(name, src))
    (OUT / "glsl/material_new.glsl").write_text(material_codegen((REF_ROOT / "src/pt/material_new.glsl").read_text()))
    trace = (REF_ROOT / "src/pt/pt_trace.comp").read_text()
    (OUT / "glsl/pt_trace_visitor.glsl").write_text(extract_trace_visitor(trace))
    (OUT / "glsl/pt_trace_geometry.glsl").write_text(extract_drawable_geometry(trace))
    (OUT / "glsl/raymarch.glsl").write_text(raymarch_to_cpp((REF_ROOT / "src/pt/raymarch.glsl").read_text()))
    (OUT / "glsl/sdf_snippets.inc").write_text(
        extract_sdf_snippets((REF_ROOT / "src/pathtracer/sdf.hpp").read_text()))
    for name in PP_SHADERS:
        (OUT / "glsl" / f"{name}.inc").write_text(pp_to_cpp(name, (REF_ROOT / "src/pt" / f"{name}.comp").read_text()))
    (OUT / "glsl/forward_resolve.inc").write_text(
        resolve_to_cpp((REF_ROOT / "src/pt/forward/resolve.frag").read_text()))
    for name in PASS_SHADERS:
        (OUT / "glsl" / f"{name}.inc").write_text(pass_to_cpp(name, (REF_ROOT / "src/pt" / f"{name}.comp").read_text()))
    (OUT / "glsl/bokeh.inc").write_text(glsl_to_cpp((REF_ROOT / "src/pt/bokeh.glsl").read_text(),
                                                    globals_thread_local=False))


def compile_ref() -> Path:
    lib = OUT / "libmyrt_ref.so"
    flags = ["-std=c++23", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fwrapv", "-fno-fast-math", "-pthread",
             "-w"]
    incs = ["-I", str(HERE / "shim"), "-I", str(REF_ROOT / "src/pathtracer"), "-I", str(REF_ROOT / "src"), "-I",
            str(OUT / "glsl"), "-I", str(HERE)]
    srcs = [str(OUT / "src/bvh.cpp"), str(REF_ROOT / "src/thread_pool.cpp"), str(HERE / "ref_harness_bvh.cpp"),
            str(HERE / "ref_harness_glsl.cpp"), str(HERE / "ref_harness_post.cpp")]
    cmd = ["g++", *flags, *incs, *srcs, "-o", str(lib)]
    subprocess.run(cmd, check=True)
    return lib


def main() -> int:
    if not (REF_ROOT / "src/pathtracer/bvh.cpp").exists():
        print(f"reference tree not found at {REF_ROOT}; oracle/_ref not rebuilt", file=sys.stderr)
        return 0
    write_sources()
    lib = compile_ref()
    print(f"built {lib}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
