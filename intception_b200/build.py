"""Build libintception_b200.so in-tree for sm_100a.

Steps: regenerate the device Boys table (mpmath), emit the per-class kernels,
compile every translation unit with nvcc in parallel, link one shared library.
Outputs: intception_b200/libintception_b200.so; objects in intception_b200/_build/.

    python -m intception_b200.build [--jobs N] [--force]
"""
import argparse
import concurrent.futures as cf
import hashlib
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, 'csrc')
GEN = os.path.join(CSRC, '_gen')
BUILD = os.path.join(PKG, '_build')
LIB = os.path.join(PKG, 'libintception_b200.so')
NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
         '-Xptxas', '-warn-spills', '-I', CSRC, '-I', os.path.join(ROOT, 'include')]


def _generate():
    sys.path.insert(0, ROOT)
    import json
    from intception_b200.emit import boys_table, eri_emitter
    boys_table.write_headers(GEN)
    stats = eri_emitter.emit_all(GEN)
    with open(os.path.join(PKG, 'class_stats.json'), 'w') as fh:
        json.dump(stats, fh, indent=0)


def _sources():
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith('.cu')]
    srcs += [os.path.join(GEN, f) for f in sorted(os.listdir(GEN)) if f.endswith('.cu')]
    return srcs


def _headers_digest():
    h = hashlib.sha1()
    for d in (CSRC, GEN, os.path.join(ROOT, 'include')):
        for f in sorted(os.listdir(d)):
            if f.endswith(('.cuh', '.h')):
                with open(os.path.join(d, f), 'rb') as fh:
                    h.update(f.encode())
                    h.update(fh.read())
    h.update(' '.join(ARCH + FLAGS).encode())
    return h.hexdigest()


def _compile(src, digest, force):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + '.o')
    stamp = obj + '.dep'
    with open(src, 'rb') as fh:
        key = hashlib.sha1(fh.read() + digest.encode()).hexdigest()
    if not force and os.path.exists(obj) and os.path.exists(stamp) and open(stamp).read() == key:
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + ['-c', src, '-o', obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed for %s:\n%s\n%s' % (src, r.stdout, r.stderr))
    with open(stamp, 'w') as fh:
        fh.write(key)
    return obj, (r.stdout + r.stderr).strip()


def build(jobs=None, force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    _generate()
    digest = _headers_digest()
    srcs = _sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    objs = []
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = {ex.submit(_compile, s, digest, force): s for s in srcs}
        for f in cf.as_completed(futs):
            obj, log = f.result()
            objs.append(obj)
            if verbose and log:
                print(log)
    objs.sort()
    newest = max(os.path.getmtime(o) for o in objs)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < newest:
        tmp = LIB + '.tmp'
        cmd = [NVCC] + ARCH + ['-shared', '-o', tmp] + objs + ['-lcudart']
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('link failed:\n%s\n%s' % (r.stdout, r.stderr))
        os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('--jobs', type=int, default=None)
    ap.add_argument('--force', action='store_true')
    ap.add_argument('-v', '--verbose', action='store_true')
    a = ap.parse_args()
    print(build(a.jobs, a.force, a.verbose))
