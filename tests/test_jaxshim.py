"""The NumPy stand-in for JAX used to run the reference's source for the golden
fixtures (``tests/golden/jaxshim``) behaves as JAX documents for the cases the
reference relies on.  Run in a subprocess so the stand-in's ``jax`` module
never enters this test session."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

SCRIPT = r'''
import numpy as np
import jax
import jax.numpy as jnp
from jax import lax
jax.config.update("jax_enable_x64", True)

x = jnp.arange(5.0)
# functional update: the original is unchanged
y = x.at[1].set(10.0)
assert float(x[1]) == 1.0 and float(y[1]) == 10.0
# out-of-bounds scatter updates are dropped, negative indices count from the end
y = x.at[np.array([-1, 7, -9])].set(np.array([5.0, 6.0, 7.0]))
assert list(np.asarray(y)) == [0.0, 1.0, 2.0, 3.0, 5.0]
# add accumulates duplicate indices
y = x.at[np.array([0, 0, 2])].add(np.array([1.0, 2.0, 3.0]))
assert list(np.asarray(y)) == [3.0, 1.0, 5.0, 3.0, 4.0]
# gathers clamp out-of-bounds indices
assert list(np.asarray(x[np.array([-1, 9, 2])])) == [4.0, 4.0, 2.0]
# immutability: augmented assignment rebinds, the other name keeps its value
a = jnp.ones(3); b = a; b += 1.0
assert float(a[0]) == 1.0 and float(b[0]) == 2.0
try:
    a[0] = 5.0
    raise SystemExit("item assignment must fail")
except TypeError:
    pass
# jit lifts NumPy arguments to jax arrays (with .at)
f = jax.jit(lambda v: v.at[0].set(-1.0))
assert float(f(np.zeros(2))[0]) == -1.0
# restriction (2x2 block sums) and prolongation (injection) as the reference calls them
r = np.random.default_rng(0).standard_normal((6, 4, 3))
k = jnp.full((2, 2, 1, 1), 1.0)
dn = lax.conv_dimension_numbers((1,) + r.shape, k.shape, ("CHWN", "HWIO", "CHWN"))
rc = np.asarray(lax.conv_general_dilated(r[None], k, (2, 2), "VALID", dimension_numbers=dn)[0])
assert np.allclose(rc, r.reshape(3, 2, 2, 2, 3).sum(axis=(1, 3)))
p = np.asarray(lax.conv_general_dilated(rc[None], k, (1, 1), ((1, 1), (1, 1)), (2, 2), (1, 1),
                                        dimension_numbers=dn)[0])
assert np.array_equal(p, rc.repeat(2, axis=0).repeat(2, axis=1))
# vmap over a trailing axis, stacked on the trailing axis
v = jax.vmap(lambda a, s: jnp.roll(a, s, axis=0), in_axes=(-1, 0), out_axes=-1)(
    jnp.asarray(np.arange(12.0).reshape(4, 3)), np.array([0, 1, 2]))
assert np.array_equal(np.asarray(v)[:, 1], np.roll(np.arange(12.0).reshape(4, 3)[:, 1], 1))
print("ok")
'''


def test_stand_in_semantics():
    env = dict(os.environ, PYTHONPATH=os.path.join(HERE, "golden", "jaxshim"), PYTHONDONTWRITEBYTECODE="1")
    r = subprocess.run([sys.executable, "-c", SCRIPT], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
