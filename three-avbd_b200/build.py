"""Builds the CUDA backend into avbd_b200/libavbd_cuda.so (in-tree, so it travels with the repo).

nvcc for sm_100a only. The collision translation unit is compiled with --fmad=false: its pair
tests and SAT choices round every operation separately, as the oracle's f32 restatement does. The
solve translation unit uses the approximate single-precision division and square root
(-prec-div=false -prec-sqrt=false, at most 2 ulp each): the solve is held to the FP64 oracle within a
tolerance, not bit for bit, and the IEEE-rounded forms were a fifth of its time.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
OUT = os.path.join(HERE, 'avbd_b200', 'libavbd_cuda.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr', '-I', CSRC,
          '-I', os.path.join(HERE, '..', 'include')]
UNITS = {
    'avbd_collide.cu': ['--fmad=false'],
    'avbd_solve.cu': ['-prec-div=false', '-prec-sqrt=false'],
    'avbd_host.cu': [],
    'avbd_batch.cu': [],
    'avbd_hull.cu': [],
    'avbd_adjoint.cu': [],
    'avbd_record.cu': [],
    'avbd_query.cu': [],
    'avbd_capture.cu': [],
}


def nvcc() -> str:
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return 'nvcc'


def _stale(out: str, deps: list) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.cuh', '.hpp'))] + [os.path.join(HERE, '..', 'include', 'avbd.h')]
    objs = []
    for unit, flags in UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(BUILD, unit.replace('.cu', '.o'))
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            cmd = [nvcc()] + ARCH + COMMON + flags + ['-c', src, '-o', obj]
            if verbose:
                cmd.insert(1, '-Xptxas=-v')
            subprocess.run(cmd, check=True)
    if force or _stale(OUT, objs):
        subprocess.run([nvcc()] + ARCH + ['-shared', '-o', OUT] + objs + ['-lcudart'], check=True)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
