#!/usr/bin/env python3
"""Build oracle/_ref/libtgref.so: the reference's own tracking kernels on the CPU.

Test infrastructure only.  For each (model, coefficient count, algorithm)
combination this script lets the reference assemble its `tractogram` kernel
exactly as it does before launching it (tractography/tracking.py:92-173):
it calls the reference's ``tracking.tractogram`` with a recording runtime
whose ``build_program`` keeps the source instead of compiling it.  The
source is then made C++: the reference's ``#include``d kernel files are
inlined from the reference tree, OpenCL vector literals ``(float4)(...)``
and ``(T){...}`` become ``make_T(...)`` calls, the templated point budget
becomes a run-time value, and one counter increment is inserted before the
orientation update so accepted steps can be counted.  oracle/clshim.hpp
supplies the OpenCL built-ins.  g++ compiles each variant in its own
translation unit and namespace; the outputs go only to oracle/_ref/.
The boundary BVH traversal (utils/bvh.cl), the boundary sampler of
domain.seed and the `tod` and `connectome` kernels (SH lmax 8, image
domain) are compiled the same way with batch drivers, for the BVH hit,
boundary-seeding, TOD and connectome parity tests.

Nothing from the reference is copied into this repository: the sources are
read from the reference tree at build time.

Usage: python oracle/build_ref.py [--reference DIR]   (default: $TG_REFERENCE_ROOT,
       else the reference checkout this recipe is set up for)
"""

from __future__ import annotations

import argparse
import os
import re
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


def reference_root() -> Path:
    """Where the reference sources are read from: $TG_REFERENCE_ROOT, else the
    checkout location of this build machine.  The recipes that read the
    reference (this one, tests/golden/make_*.py, oracle/step_error.py) share it."""
    return Path(os.environ.get("TG_REFERENCE_ROOT", "/root/reference"))
N_STEPS_SENTINEL = 987654
NNZ_SENTINEL = 54321     # nonzero voxels of the FOD the seeding kernel is captured with

VARIANTS = [
    # name, model, coefficients, algorithm
    ("sh15_transport", "sh", 15, "transport"),
    ("sh15_diffusion", "sh", 15, "diffusion"),
    ("sh28_transport", "sh", 28, "transport"),
    ("sh28_diffusion", "sh", 28, "diffusion"),
    ("sh45_transport", "sh", 45, "transport"),
    ("sh45_diffusion", "sh", 45, "diffusion"),
    ("dti_transport", "dti", 6, "transport"),
    ("dti_diffusion", "dti", 6, "diffusion"),
]


class _Captured(Exception):
    pass


class RecordingRuntime:
    """Stands in for OpenCLRuntime: records the program source, runs nothing."""

    def __init__(self):
        self.source = None

    def buffer_from_array(self, data, access=None):
        return np.ascontiguousarray(data)

    def allocate_buffer(self, nbytes, access=None):
        return nbytes

    def build_program(self, source, options=()):
        self.source = source
        raise _Captured()

    def build_kernel_program(self, names, values=None, *, options=()):
        # the reference's own loader and templating (opencl.py:86-109), which
        # ends in build_program above
        return sys.modules["tractography.opencl"].OpenCLRuntime.build_kernel_program(
            self, names, values, options=options)


def capture(ref, model, n_coefficients, algorithm):
    Image = sys.modules["nibabel.nifti1"].Nifti1Image
    field = ref.field.Image(Image(np.ones((2, 2, 2, n_coefficients), np.float32), np.eye(4)))
    domain = ref.domain.Image(Image(np.ones((2, 2, 2), np.uint8), np.eye(4)))
    local = ref.local.DiffusionTensorImaging() if model == "dti" else \
        ref.local.RealSymmetricSphericalHarmonics(n_coefficients)
    alg = ref.algorithm.Transport(local) if algorithm == "transport" else ref.algorithm.Diffusion(local)
    seeds = np.array([[0, 0, 0, 1, 1, 0, 0, 0]], np.float32)
    rt = RecordingRuntime()
    try:
        ref.tracking.tractogram(alg, domain, field, seeds, save_at=1.0,
                                maximum_streamline_length=float(N_STEPS_SENTINEL), runtime=rt)
    except _Captured:
        return rt.source
    raise RuntimeError("the reference did not build a program")


def capture_update(ref, model, n_coefficients, algorithm):
    """The reference's standalone orientation-update kernel (algorithm.py:701-790)."""
    local = ref.local.DiffusionTensorImaging() if model == "dti" else \
        ref.local.RealSymmetricSphericalHarmonics(n_coefficients)
    alg = ref.algorithm.Transport(local) if algorithm == "transport" else ref.algorithm.Diffusion(local)
    rt = RecordingRuntime()
    try:
        ref.algorithm.update_orientation(alg, np.zeros((1, n_coefficients)), np.array([[0.0, 0.0, 1.0]]), runtime=rt)
    except _Captured:
        return rt.source
    raise RuntimeError("the reference did not build a program")


def inline_includes(text, kernel_dir, seen=None):
    seen = set() if seen is None else seen

    def repl(m):
        path = kernel_dir / m.group(1)
        if path in seen:
            return ""
        seen.add(path)
        return inline_includes(path.read_text(), kernel_dir, seen)

    return re.sub(r'#include\s+"([^"]+)"', repl, text)


def rewrite_literals(text):
    # (T)(...)  ->  make_T(...)
    text = re.sub(r"\((float|int|uint)([234])\)\s*\(", r"make_\1\2(", text)
    # (T){...}  ->  make_T(...) for vectors, T{...} for structs
    out = []
    i = 0
    pattern = re.compile(r"\((float|int|uint)([234])\)\s*\{|\((ModelValue|model_value_t)\)\s*\{")
    while True:
        m = pattern.search(text, i)
        if not m:
            out.append(text[i:])
            break
        out.append(text[i:m.start()])
        depth, j = 1, m.end()
        while depth:
            depth += {"{": 1, "}": -1}.get(text[j], 0)
            j += 1
        inner = text[m.end():j - 1]
        if m.group(1):
            out.append(f"make_{m.group(1)}{m.group(2)}({inner})")
        else:
            out.append(f"{m.group(3)}{{{inner}}}")
        i = j
    return "".join(out)


def to_cpp(source, kernel_dir, name):
    text = inline_includes(source, kernel_dir)
    text = rewrite_literals(text)
    text = text.replace(str(N_STEPS_SENTINEL), "tgref_n_steps")
    text = text.replace("orientation = algorithm_update_orientation(",
                        "++tgref_steps; orientation = algorithm_update_orientation(")
    # algorithm.py:219 draws two normals inside one expression; C leaves the
    # order of the two calls unspecified.  clang (pocl, the reference's CI
    # platform) evaluates them left to right, g++ right to left: sequence them
    # left to right explicitly so this build draws what the reference draws.
    text = re.sub(r"noise\s*=\s*randn\(rng_state\)\s*\*\s*et\s*\+\s*randn\(rng_state\)\s*\*\s*ep\s*;",
                  "{ const float tgref_n1 = randn(rng_state); const float tgref_n2 = randn(rng_state); "
                  "noise = tgref_n1 * et + tgref_n2 * ep; }", text)
    return (f'#include "clshim.hpp"\n'
            f"extern unsigned int tgref_n_steps;\n"
            f"extern thread_local unsigned long long tgref_steps;\n"
            f"namespace {name} {{\n{text}\n}}\n")


DRIVER = """
extern "C" unsigned long long tgref_{name}(const int* mask, const unsigned int* mdims, const float* minv,
        const float* field, const unsigned int* fdims, const float* finv, float step, float gamma, float noise,
        unsigned int rng_seed, const float* seeds, unsigned int n_seeds, float* out, unsigned int* lengths,
        float save_at, unsigned int n_steps, int threads)
{{
    tgref_n_steps = n_steps;
    const float4 dummy4 = make_float4(0.0f);
    const uint4 dummyu4 = make_uint4(0u);
    const int4 dummyi4 = make_int4(0);
    const float dummyf = 0.0f;
    const unsigned int dummyu = 0;
    unsigned long long total = 0;
    long g;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total) num_threads(threads > 0 ? threads : 1)
    for (g = 0; g < (long)n_seeds; ++g) {{
        tgref_global_id = (size_t)g;
        tgref_steps = 0;
        {name}::tractogram(&dummy4, &dummyu4, &dummyf, 1u, &dummy4, &dummy4, &dummyi4, &dummyu, 1u,
            mask, make_uint3(mdims[0], mdims[1], mdims[2]), (const float4*)minv,
            field, make_uint4(fdims[0], fdims[1], fdims[2], fdims[3]), (const float4*)finv,
            step, gamma{noise_arg}, rng_seed, (const float4*)seeds, n_seeds, (float4*)out, lengths, save_at);
        total += tgref_steps;
    }}
    return total;
}}
"""


UPDATE_DRIVER = """
extern "C" void tgref_update_{name}(float step, float gamma, float noise, unsigned int rng_seed,
        const float* params, const float* orientations, unsigned int n, float* out)
{{
    for (unsigned int g = 0; g < n; ++g) {{
        tgref_global_id = g;
        {name}::update_orientation(step, gamma{noise_arg}, rng_seed, params, (const float4*)orientations, n,
                                   (float4*)out);
    }}
}}
"""


BVH_DRIVER = """
extern "C" void tgref_bvh_hits(const float* vertices, const unsigned int* triangles, const float* bounds_min,
        const float* bounds_max, const int* nodes, const unsigned int* ordered, unsigned int n_nodes,
        const float* starts, const float* ends, unsigned int n, unsigned char* found, unsigned int* triangle,
        float* hit)
{
    const bvhref::BVH bvh = {(const float4*)vertices, (const uint4*)triangles, (const float4*)bounds_min,
                             (const float4*)bounds_max, (const int4*)nodes, ordered, n_nodes};
    for (unsigned int i = 0; i < n; ++i) {
        const float3 s = make_float3(starts[4 * i], starts[4 * i + 1], starts[4 * i + 2]);
        const float3 e = make_float3(ends[4 * i], ends[4 * i + 1], ends[4 * i + 2]);
        unsigned int tri = 0;
        float3 bc = make_float3(0.0f, 0.0f, 0.0f);
        float t = 1.0f;
        found[i] = bvhref::bvh_segment_hit(bvh, s, e, &tri, &bc, &t) ? 1 : 0;
        triangle[i] = tri;
        hit[4 * i] = bc.x;
        hit[4 * i + 1] = bc.y;
        hit[4 * i + 2] = bc.z;
        hit[4 * i + 3] = t;
    }
}
"""


SEED_DRIVER = """
extern "C" void tgref_boundary_seeds(const float* vertices, const unsigned int* triangles, const float* cumulative,
        unsigned int n_triangles, unsigned int rng_seed, unsigned int n, float* locations, float* orientations)
{
    const float4 dummy4[4] = {make_float4(0.0f), make_float4(0.0f), make_float4(0.0f), make_float4(0.0f)};
    const int4 dummyi4 = make_int4(0);
    const unsigned int dummyu = 0;
    const int mask = 1;
    for (unsigned int g = 0; g < n; ++g) {
        tgref_global_id = g;
        seedref::sample_domain_boundary((const float4*)vertices, (const uint4*)triangles, cumulative, n_triangles,
            dummy4, dummy4, &dummyi4, &dummyu, 0u, &mask, make_uint3(1u, 1u, 1u), dummy4, rng_seed, n,
            (float4*)locations, (float4*)orientations);
    }
}
"""


def capture_seed(ref):
    """The boundary sampler kernel the reference assembles in domain.seed (domain.py:494-575)."""
    Image = sys.modules["nibabel.nifti1"].Nifti1Image
    domain = ref.domain.Image(Image(np.ones((2, 2, 2), np.uint8), np.eye(4)))
    rt = RecordingRuntime()
    try:
        ref.domain.seed(domain, 4, rng_seed=1, runtime=rt)
    except _Captured:
        return rt.source
    raise RuntimeError("the reference did not build a program")


PRODUCT_VARIANTS = [("sh45_transport", "transport"), ("sh45_diffusion", "diffusion")]

TOD_DRIVER = """
extern "C" void tgref_{name}(const float* bv, const unsigned int* bi, const float* bc, unsigned int n_tri,
        const float* bmin, const float* bmax, const int* nodes, const unsigned int* ordered, unsigned int n_nodes,
        const int* mask, const unsigned int* mdims, const float* minv, const float* field, const unsigned int* fdims,
        const float* finv, float step, float gamma, float noise, unsigned int rng_seed, unsigned int n_seeds,
        unsigned int n_steps, const unsigned int* odims, const float* oinv, float* coefficients, int threads)
{{
    (void)noise;
    tgref_n_steps = n_steps;
    long g;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
    for (g = 0; g < (long)n_seeds; ++g) {{
        tgref_global_id = (size_t)g;
        {name}::tod((const float4*)bv, (const uint4*)bi, bc, n_tri, (const float4*)bmin, (const float4*)bmax,
            (const int4*)nodes, ordered, n_nodes, mask, make_uint3(mdims[0], mdims[1], mdims[2]), (const float4*)minv,
            field, make_uint4(fdims[0], fdims[1], fdims[2], fdims[3]), (const float4*)finv, step, gamma{noise_arg},
            rng_seed, n_seeds, make_uint4(odims[0], odims[1], odims[2], 0u), (const float4*)oinv, coefficients);
    }}
}}
"""

CONNECTOME_DRIVER = """
extern "C" void tgref_{name}(const float* bv, const unsigned int* bi, const float* bc, unsigned int n_tri,
        const float* bmin, const float* bmax, const int* nodes, const unsigned int* ordered, unsigned int n_nodes,
        const int* mask, const unsigned int* mdims, const float* minv, const float* field, const unsigned int* fdims,
        const float* finv, float step, float gamma, float noise, unsigned int rng_seed, unsigned int n_seeds,
        unsigned int n_steps, float minimum_length, int* rows, int* columns, float* weights, int threads)
{{
    (void)noise;
    tgref_n_steps = n_steps;
    long g;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
    for (g = 0; g < (long)n_seeds; ++g) {{
        tgref_global_id = (size_t)g;
        {name}::connectome((const float4*)bv, (const uint4*)bi, bc, n_tri, (const float4*)bmin, (const float4*)bmax,
            (const int4*)nodes, ordered, n_nodes, mask, make_uint3(mdims[0], mdims[1], mdims[2]),
            (const float4*)minv, field, make_uint4(fdims[0], fdims[1], fdims[2], fdims[3]), (const float4*)finv,
            step, gamma{noise_arg}, rng_seed, n_seeds, minimum_length, rows, columns, weights);
    }}
}}
"""


def _product_objects(ref, algorithm):
    Image = sys.modules["nibabel.nifti1"].Nifti1Image
    field = ref.field.Image(Image(np.ones((2, 2, 2, 45), np.float32), np.eye(4)))
    domain = ref.domain.Image(Image(np.ones((2, 2, 2), np.uint8), np.eye(4)))
    local = ref.local.RealSymmetricSphericalHarmonics(45)
    alg = ref.algorithm.Transport(local, step_size=1.0) if algorithm == "transport" else \
        ref.algorithm.Diffusion(local, step_size=1.0)
    return field, domain, alg, Image


def capture_tod(ref, algorithm):
    """The reference's `tod` kernel source (tracking.py:255-356)."""
    field, domain, alg, Image = _product_objects(ref, algorithm)
    rt = RecordingRuntime()
    try:
        ref.tracking.tod(alg, domain, field, Image(np.zeros((2, 2, 2), np.float32), np.eye(4)), 1,
                         maximum_streamline_length=float(N_STEPS_SENTINEL), runtime=rt)
    except _Captured:
        return rt.source
    raise RuntimeError("the reference did not build a program")


def capture_connectome(ref, algorithm):
    """The reference's `connectome` kernel source (tracking.py:458-553)."""
    field, domain, alg, _ = _product_objects(ref, algorithm)
    rt = RecordingRuntime()
    try:
        ref.tracking.connectome(alg, domain, field, 1, maximum_streamline_length=float(N_STEPS_SENTINEL), runtime=rt)
    except _Captured:
        return rt.source
    raise RuntimeError("the reference did not build a program")


FOD_SEED_VARIANTS = [("fodseed_sh45", "sh", 45), ("fodseed_dti", "dti", 6)]

FOD_SEED_DRIVER = """
extern "C" void tgref_{name}(const float* fod, const float* voxels, const float* affine, unsigned int* states,
        float* seeds, unsigned int nnz, unsigned int n, int threads)
{{
    tgref_nnz = nnz;
    long g;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
    for (g = 0; g < (long)n; ++g) {{
        tgref_global_id = (size_t)g;
        {name}::seeds_from_fod((const float (*)[{C}])fod, (const float4*)voxels, (const float4*)affine,
                               (uint2*)states, (float4 (*)[2])seeds);
    }}
}}
"""


def capture_fod_seeds(ref, n_coefficients):
    """The FOD seeding kernel as seeds.from_fod assembles it (seeds.py:174-216,
    utils/seeds.cl), for a volume of NNZ_SENTINEL nonzero voxels."""
    Image = sys.modules["nibabel.nifti1"].Nifti1Image
    fod = Image(np.ones((NNZ_SENTINEL, 1, 1, n_coefficients), np.float32), np.eye(4))
    rt = RecordingRuntime()
    state = np.random.get_state()
    try:
        ref.seeds.from_fod(fod, 4, runtime=rt)
    except _Captured:
        return rt.source
    finally:
        np.random.set_state(state)
    raise RuntimeError("the reference did not build a program")


def fod_seed_source(ref, kernel_dir, name, n_coefficients):
    src = capture_fod_seeds(ref, n_coefficients)
    # the voxel count is a template value in the kernel (randi(state, $nnz));
    # make it the driver's run-time value (array bounds keep the sentinel,
    # they are pointers once the kernel is compiled)
    call = f"randi(state, {NNZ_SENTINEL})"
    if src.count(call) != 1:
        raise RuntimeError("unexpected seeding kernel source")
    src = src.replace(call, "randi(state, tgref_nnz)")
    cpp = to_cpp(src, kernel_dir, name).replace("extern unsigned int tgref_n_steps;",
                                                  "extern unsigned int tgref_nnz;")
    # utils/seeds.cl:94 draws the x, y and z jitter inside one vector
    # literal; as make_float4 arguments g++ would draw them right to left, so
    # sequence them left to right as clang (pocl) evaluates the initialiser
    jitter = re.compile(r"voxel\s*\+=\s*make_float4\(randu\(state\)\s*-\s*0\.5f,\s*randu\(state\)\s*-\s*0\.5f,"
                        r"\s*randu\(state\)\s*-\s*0\.5f,\s*0\.0f\);")
    cpp, n = jitter.subn("{ const float tgref_j0 = randu(state) - 0.5f; const float tgref_j1 = randu(state) - 0.5f; "
                         "const float tgref_j2 = randu(state) - 0.5f; voxel += make_float4(tgref_j0, tgref_j1, "
                         "tgref_j2, 0.0f); }", cpp)
    if n != 1:
        raise RuntimeError("unexpected seeding kernel source (jitter draw)")
    return cpp + FOD_SEED_DRIVER.format(name=name, C=n_coefficients)


def bvh_source(kernel_dir):
    """utils/bvh.cl (the boundary BVH traversal) as C++ with a batch driver."""
    text = rewrite_literals(inline_includes((kernel_dir / "utils" / "bvh.cl").read_text(), kernel_dir))
    return f'#include "clshim.hpp"\nnamespace bvhref {{\n{text}\n}}\n' + BVH_DRIVER


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(reference_root()))
    args = ap.parse_args()
    reference = Path(args.reference)
    sys.path.insert(0, str(HERE.parent))
    from oracle.refstubs import install_stubs

    install_stubs(reference)
    import tractography as ref  # the reference package

    kernel_dir = reference / "tractography" / "resources" / "kernels"
    OUT.mkdir(exist_ok=True)
    objects = []
    common = OUT / "tgref_common.cpp"
    common.write_text('#include <cstddef>\nthread_local size_t tgref_global_id;\nunsigned int tgref_n_steps;\n'
                      'thread_local unsigned long long tgref_steps;\nunsigned int tgref_nnz;\n')
    sources = [common]
    for name, model, C, algorithm in VARIANTS:
        src = capture(ref, model, C, algorithm)
        cpp = to_cpp(src, kernel_dir, name)
        cpp += DRIVER.format(name=name, noise_arg=", noise" if algorithm == "diffusion" else "")
        path = OUT / f"tgref_{name}.cpp"
        path.write_text(cpp)
        sources.append(path)
        uname = "u_" + name
        ucpp = to_cpp(capture_update(ref, model, C, algorithm), kernel_dir, uname)
        ucpp += UPDATE_DRIVER.format(name=uname, noise_arg=", noise" if algorithm == "diffusion" else "")
        upath = OUT / f"tgref_{uname}.cpp"
        upath.write_text(ucpp)
        sources.append(upath)
    bpath = OUT / "tgref_bvh.cpp"
    bpath.write_text(bvh_source(kernel_dir))
    sources.append(bpath)
    for name, algorithm in PRODUCT_VARIANTS:
        noise_arg = ", noise" if algorithm == "diffusion" else ""
        for kind, capture_fn, driver in (("tod", capture_tod, TOD_DRIVER),
                                         ("connectome", capture_connectome, CONNECTOME_DRIVER)):
            tname = f"{kind}_{name}"
            path = OUT / f"tgref_{tname}.cpp"
            path.write_text(to_cpp(capture_fn(ref, algorithm), kernel_dir, tname) +
                            driver.format(name=tname, noise_arg=noise_arg))
            sources.append(path)
    for name, _model, C in FOD_SEED_VARIANTS:
        path = OUT / f"tgref_{name}.cpp"
        path.write_text(fod_seed_source(ref, kernel_dir, name, C))
        sources.append(path)
    spath = OUT / "tgref_seed.cpp"
    spath.write_text(to_cpp(capture_seed(ref), kernel_dir, "seedref").replace(
        "extern unsigned int tgref_n_steps;", "") + SEED_DRIVER)
    sources.append(spath)
    flags = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off", "-march=x86-64-v3",
             "-mtune=generic", "-w", f"-I{HERE}"]
    procs = []
    for src in sources:
        obj = src.with_suffix(".o")
        objects.append(obj)
        # OpenCL C passes `const float fod[]` to a `float*` parameter
        # (utils/seeds.cl:40 into the models' evaluate_interpolated_model);
        # C++ needs -fpermissive to accept that conversion
        extra = ["-fpermissive"] if src.name.startswith("tgref_fodseed_") else []
        procs.append(subprocess.Popen(["g++", *flags, *extra, "-c", str(src), "-o", str(obj)]))
    if any(p.wait() != 0 for p in procs):
        raise SystemExit("compiling the reference kernels failed")
    subprocess.run(["g++", "-shared", "-fopenmp", "-o", str(OUT / "libtgref.so"), *map(str, objects)], check=True)
    print(f"built {OUT / 'libtgref.so'} ({len(VARIANTS)} kernel variants)")


if __name__ == "__main__":
    main()
