"""Generate golden_noise.npz from the REFERENCE's stochastic Kraus channels.

Run here (the reference checkout is not present on a GPU box):

    python tests/golden/make_noise_golden.py --reference PATH_OF_REFERENCE_CHECKOUT

It imports the reference's ``dense_evolution/noise/kraus_channels.py`` and
``dense_evolution/noise/kraus/*.py`` unmodified.  JAX is absent from this image,
so ``jax`` is replaced by a stub whose array type matches nothing: every
channel then takes its NumPy branch, which is deterministic for a seeded
``np.random.Generator`` (one fire/no-fire draw per qubit per call, index bit q
for qubit q).  Each case records the input state, the model, p, the qubit
subset, the seed and the reference's output state.
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def load_noise(root: str):
    pkg_root = os.path.join(root, 'dense_evolution')
    for name, sub in [('dense_evolution', ''), ('dense_evolution.noise', 'noise'),
                      ('dense_evolution.noise.kraus', os.path.join('noise', 'kraus'))]:
        m = types.ModuleType(name)
        m.__path__ = [os.path.join(pkg_root, sub) if sub else pkg_root]
        sys.modules[name] = m
    jax = types.ModuleType('jax')
    jnp = types.ModuleType('jax.numpy')

    class _NoJaxArray:          # nothing is an instance: the NumPy branch always runs
        pass
    jnp.ndarray = _NoJaxArray
    jax.numpy = jnp
    errors = types.ModuleType('jax.errors')
    errors.TracerBoolConversionError = type('TracerBoolConversionError', (Exception,), {})
    jax.errors = errors
    sys.modules['jax'] = jax
    sys.modules['jax.numpy'] = jnp
    sys.modules['jax.errors'] = errors
    return importlib.import_module('dense_evolution.noise.kraus_channels').NoiseModel


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', required=True, help='path of the reference checkout')
    args = ap.parse_args()
    NoiseModel = load_noise(args.reference)
    rng0 = np.random.default_rng(77)
    out = {}
    k = 0
    for model in NoiseModel.MODELS:
        for n, p, qubits in [(5, 0.35, None), (6, 0.8, [0, 2, 5]), (4, 0.0, None), (7, 0.5, None)]:
            for seed in (1, 2):
                v = rng0.normal(size=1 << n) + 1j * rng0.normal(size=1 << n)
                v /= np.linalg.norm(v)
                res = NoiseModel.apply_to_sv(v.copy(), n, model, p, rng=np.random.default_rng(seed),
                                             qubits=qubits)
                out[f'c{k}_in'] = v
                out[f'c{k}_out'] = np.asarray(res, dtype=np.complex128)
                out[f'c{k}_meta'] = np.array([n, p, seed, NoiseModel.MODELS.index(model)], dtype=np.float64)
                out[f'c{k}_qubits'] = np.array(qubits if qubits is not None else [], dtype=np.int64)
                out[f'c{k}_hasq'] = np.array([qubits is not None])
                k += 1
    out['ncases'] = np.array([k])
    out['models'] = np.array(NoiseModel.MODELS)
    np.savez_compressed(os.path.join(HERE, 'golden_noise.npz'), **out)
    print(f'{k} cases -> golden_noise.npz')


if __name__ == '__main__':
    main()
