"""Build libgsb.so (the CUDA kernels and the C ABI of include/gsb.h) in-tree for sm_100a.

    python -m galsim_b200.build          # or galsim_b200.build.build()

The shared library is written next to this file so that it travels with the repository
checkout; nothing is installed into site-packages and there is no JIT cache.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIB = os.path.join(HERE, 'libgsb.so')
SOURCES = ['gsb_api.cu', 'gsb_tables.cu', 'gsb_draw.cu', 'gsb_draw_f32_small.cu',
           'gsb_draw_f32_large.cu', 'gsb_draw_f64_small.cu', 'gsb_draw_f64_large.cu', 'gsb_draw_large.cu',
           'gsb_noalloc.cu', 'gsb_adjoint.cu', 'gsb_adjoint_f32_small.cu', 'gsb_adjoint_f32_large.cu',
           'gsb_adjoint_f64_small.cu', 'gsb_adjoint_f64_large.cu', 'gsb_adjoint_large.cu', 'gsb_images.cu', 'gsb_noise.cu',
           'gsb_fits.cu', 'gsb_standalone.cu', 'gsb_chromatic.cu', 'gsb_real.cu']
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return 'nvcc'


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, 'include', 'gsb.h')]
    if any(os.path.getmtime(d) > t for d in deps):
        return True
    # a source added since the library was linked, or an object older than its source
    build_dir = os.path.join(HERE, '_build')
    for src in SOURCES:
        obj = os.path.join(build_dir, src.replace('.cu', '.o'))
        if os.path.isdir(build_dir) and (not os.path.exists(obj) or
                                         os.path.getmtime(obj) < os.path.getmtime(os.path.join(CSRC, src))):
            return True
    return False


def build(force=False, verbose=False):
    """Compile the sources into galsim_b200/libgsb.so if any is newer than the library."""
    if not force and not _stale():
        return LIB
    objs = []
    build_dir = os.path.join(HERE, '_build')
    os.makedirs(build_dir, exist_ok=True)
    procs = []
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cuh')] + \
        [os.path.join(ROOT, 'include', 'gsb.h'), os.path.abspath(__file__)]
    newest_header = max(os.path.getmtime(h) for h in headers)
    for src in SOURCES:
        obj = os.path.join(build_dir, src.replace('.cu', '.o'))
        objs.append(obj)
        # an object is rebuilt when it is older than its source or than any header
        if (not force and os.path.exists(obj) and
                os.path.getmtime(obj) >= max(os.path.getmtime(os.path.join(CSRC, src)), newest_header)):
            continue
        cmd = [nvcc(), *ARCH, '-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC',
               '-I', os.path.join(ROOT, 'include'), '-I', CSRC, '-c', os.path.join(CSRC, src), '-o', obj]
        if verbose:
            cmd.insert(1, '-Xptxas=-v')
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0 or verbose:
            sys.stderr.write(out.decode())
        if p.returncode != 0:
            raise RuntimeError('nvcc failed: ' + ' '.join(cmd))
    tmp = LIB + '.tmp'
    subprocess.check_call([nvcc(), *ARCH, '-shared', '-o', tmp, *objs, '-lcudart'])
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose='-v' in sys.argv)
    print(LIB)
