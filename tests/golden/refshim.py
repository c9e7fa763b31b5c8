"""Run the reference pymdp's own JAX-semantics code on NumPy float64.

JAX is not installed where the golden fixtures are generated, so this module
installs small stand-in modules (``jax``, ``jax.numpy``, ``jax.lax`` ...,
``equinox``, ``opt_einsum``, ``multimethod``, ``matplotlib.pyplot``) that map
the few JAX primitives the hot path uses onto NumPy:

* ``jax.numpy``            -> ``numpy`` (float64 everywhere)
* ``lax.scan``             -> a Python loop over ``xs``
* ``vmap``                 -> a Python loop over the mapped axis + ``np.stack``
* ``tree_util.tree_map``   -> recursive map over lists / tuples / dicts
* ``nn.softmax``           -> ``exp(x - max) / sum``, the formula jax.nn uses
* ``opt_einsum.contract``  -> ``np.einsum`` in sublist form
* ``jit``                  -> identity
* array creation           -> ndarrays whose ``+=`` rebinds, as JAX's do
* ``jaxtyping`` names       -> ``numpy.ndarray`` (annotations only)

It then loads ``pymdp/utils.py``, ``pymdp/maths.py``, ``pymdp/algos.py`` and
``pymdp/control.py`` from the reference checkout unchanged, with a stand-in
``pymdp.ffi`` whose gates return False, so every call takes the pure-JAX
branch (the branch the reference's CI exercises).

This is test infrastructure: only ``tests/golden/make_golden.py`` imports it,
in a container that has the reference checkout.
"""

from __future__ import annotations

import functools
import importlib.util
import sys
import types

import numpy as np
import scipy.special as sps


def _is_leaf(x):
    return not isinstance(x, (list, tuple, dict)) and x is not None


def _tree_map(f, tree, *rest, is_leaf=None):
    if tree is None:
        return None
    if is_leaf is not None and is_leaf(tree):
        return f(tree, *rest)
    if isinstance(tree, (list, tuple)):
        out = [_tree_map(f, t, *[r[i] for r in rest], is_leaf=is_leaf) for i, t in enumerate(tree)]
        if hasattr(tree, "_fields"):  # NamedTuple
            return type(tree)(*out)
        return type(tree)(out) if isinstance(tree, tuple) else out
    if isinstance(tree, dict):
        return {k: _tree_map(f, v, *[r[k] for r in rest], is_leaf=is_leaf) for k, v in tree.items()}
    return f(tree, *rest)


def _tree_leaves(tree):
    if tree is None:
        return []
    if isinstance(tree, (list, tuple)):
        return [l for t in tree for l in _tree_leaves(t)]
    if isinstance(tree, dict):
        return [l for k in tree for l in _tree_leaves(tree[k])]
    return [tree]


def _tree_reduce(f, tree, initializer=None):
    leaves = _tree_leaves(tree)
    if initializer is None:
        return functools.reduce(f, leaves)
    return functools.reduce(f, leaves, initializer)


def _scan(f, init, xs=None, length=None):
    carry = init
    ys = []
    n = length if xs is None else len(xs)
    for i in range(n):
        carry, y = f(carry, None if xs is None else xs[i])
        ys.append(y)
    if not ys or ys[0] is None:
        return carry, None
    return carry, _tree_map(lambda *leaves: np.stack(leaves), ys[0], *ys[1:])


def _vmap(fn, in_axes=0, out_axes=0):
    def mapped(*args, **kwargs):
        axes = in_axes if isinstance(in_axes, (list, tuple)) else [in_axes] * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is None:
                continue
            for leaf in _tree_leaves(a):
                n = np.shape(leaf)[ax]
                break
            if n is not None:
                break
        if n == 0:  # an empty mapped axis: JAX returns empty outputs of the per-element shape
            probe = [a if ax is None else _tree_map(lambda x, ax=ax: np.zeros(np.delete(np.shape(x), ax)), a)
                     for a, ax in zip(args, axes)]
            with np.errstate(all="ignore"):
                out = fn(*probe, **kwargs)
            return _tree_map(lambda leaf: np.zeros((0,) + np.shape(leaf)), out)
        outs = []
        for i in range(n):
            sl = [a if ax is None else _tree_map(lambda x, ax=ax: np.take(x, i, axis=ax), a)
                  for a, ax in zip(args, axes)]
            outs.append(fn(*sl, **kwargs))
        return _tree_map(lambda *leaves: np.stack([np.asarray(l) for l in leaves]), outs[0], *outs[1:])
    return mapped


def _associative_scan(fn, elems, reverse=False, axis=0):
    """``lax.associative_scan`` as a left fold in time order:
    ``out[i] = fn(out[i - 1], elems[i])`` (the same result for an associative
    ``fn``; JAX evaluates it as a tree). ``fn`` sees a leading axis of 1, as it
    would see a batch of pairs."""
    if axis != 0:
        raise NotImplementedError("associative_scan over axis != 0")
    n = np.shape(_tree_leaves(elems)[0])[0]
    take = lambda i: _tree_map(lambda x: np.asarray(x)[i], elems)  # noqa: E731
    expand = lambda t: _tree_map(lambda x: np.asarray(x)[None], t)  # noqa: E731
    squeeze = lambda t: _tree_map(lambda x: np.asarray(x)[0], t)  # noqa: E731
    out, acc = [None] * n, None
    for i in (range(n - 1, -1, -1) if reverse else range(n)):
        cur = take(i)
        acc = cur if acc is None else squeeze(fn(expand(acc), expand(cur)))
        out[i] = acc
    return _tree_map(lambda *leaves: np.stack(leaves), out[0], *out[1:])


def _cond(pred, true_fn, false_fn, *operands, operand=None):
    """``lax.cond`` evaluated eagerly (the predicate is a concrete value)."""
    args = operands if operands else (() if operand is None else (operand,))
    return true_fn(*args) if bool(pred) else false_fn(*args)


def _jit(fn=None, **_kw):
    if fn is None:
        return lambda f: f
    return fn


def _softmax(x, axis=-1):
    x = np.asarray(x, dtype=np.float64)
    e = np.exp(x - np.max(x, axis=axis, keepdims=True))
    return e / np.sum(e, axis=axis, keepdims=True)


def _one_hot(x, n, dtype=np.float64, axis=-1):
    out = (np.asarray(x)[..., None] == np.arange(n)).astype(dtype)
    return out if axis == -1 else np.moveaxis(out, -1, axis)


def _contract(*args, backend=None, **_kw):
    conv = [list(a) if isinstance(a, tuple) else a for a in args]
    return np.einsum(*conv)


class _Multimethod:
    """First-registered implementation wins (dense arrays only here)."""

    _registry: dict = {}

    def __new__(cls, fn):
        key = (fn.__module__, fn.__name__)
        first = cls._registry.setdefault(key, fn)

        @functools.wraps(first)
        def call(*a, **k):
            return first(*a, **k)

        return call


class _ImmutableStyleArray(np.ndarray):
    """ndarray whose augmented assignments rebind instead of mutating.

    JAX arrays are immutable, so ``x += y`` in reference code means
    ``x = x + y`` (broadcasting allowed, aliases untouched).
    """

    def __iadd__(self, other):
        return np.add(self, other)

    def __isub__(self, other):
        return np.subtract(self, other)

    def __imul__(self, other):
        return np.multiply(self, other)

    def __itruediv__(self, other):
        return np.true_divide(self, other)


def _immutable(fn):
    @functools.wraps(fn)
    def wrapped(*a, **k):
        out = fn(*a, **k)
        return out.view(_ImmutableStyleArray) if isinstance(out, np.ndarray) else out
    return wrapped


def _clip(a, a_min=None, a_max=None, *, min=None, max=None):  # noqa: A002
    lo = a_min if min is None else min
    hi = a_max if max is None else max
    return np.clip(a, lo, hi)


def _module(name, **attrs):
    mod = types.ModuleType(name)
    for k, v in attrs.items():
        setattr(mod, k, v)
    sys.modules[name] = mod
    return mod


def install_shims():
    """Register the stand-in modules in ``sys.modules`` (idempotent)."""
    if "jax" in sys.modules and getattr(sys.modules["jax"], "_refshim", False):
        return
    jnp = _module("jax.numpy")
    for name in dir(np):
        if not name.startswith("_"):
            setattr(jnp, name, getattr(np, name))
    for name in ("zeros", "ones", "zeros_like", "ones_like", "full", "empty", "array",
                 "asarray", "arange", "eye", "stack", "concatenate"):
        setattr(jnp, name, _immutable(getattr(np, name)))
    jnp.clip = _immutable(_clip)
    jnp.matmul = lambda a, b, precision=None: np.matmul(a, b)
    tree_util = _module("jax.tree_util", tree_map=_tree_map, tree_reduce=_tree_reduce,
                        tree_leaves=_tree_leaves, Partial=functools.partial)
    nn = _module("jax.nn", softmax=_softmax, one_hot=_one_hot,
                 log_softmax=lambda x, axis=-1: np.log(_softmax(x, axis)))
    lax = _module("jax.lax", scan=_scan, cond=_cond, associative_scan=_associative_scan, stop_gradient=lambda x: x,
                  Precision=types.SimpleNamespace(HIGHEST=None, DEFAULT=None))
    random = _module("jax.random")
    special = _module("jax.scipy.special", xlogy=sps.xlogy, digamma=sps.digamma, gammaln=sps.gammaln)
    jscipy = _module("jax.scipy", special=special)

    class _Sparse:  # never instantiated on the dense path
        pass

    base = _module("jax.experimental.sparse._base", JAXSparse=_Sparse)
    sparse = _module("jax.experimental.sparse", BCOO=_Sparse, _base=base,
                     sparsify=lambda f: f, todense=lambda x: x)
    experimental = _module("jax.experimental", sparse=sparse)
    jax = _module("jax", numpy=jnp, tree_util=tree_util, nn=nn, lax=lax, random=random,
                  scipy=jscipy, experimental=experimental, jit=_jit, vmap=_vmap,
                  grad=None, _refshim=True)
    jax.Array = np.ndarray
    _module("equinox", Module=object, field=lambda default=None, **_k: default,
            error_if=lambda x, *a, **k: x, tree_at=None)
    jt = _module("jaxtyping")
    jt.__getattr__ = lambda name: np.ndarray
    _module("opt_einsum", contract=_contract)
    _module("multimethod", multimethod=_Multimethod)
    mpl = _module("matplotlib")
    mpl.pyplot = _module("matplotlib.pyplot")


def load_reference(ref_root: str, modules=("utils", "maths", "algos", "control")):
    """Load the reference's utils/maths/algos/control modules on the shims.

    Returns a namespace with attributes ``utils``, ``maths``, ``algos``,
    ``control``.
    """
    install_shims()
    pkg = types.ModuleType("pymdp")
    pkg.__path__ = [f"{ref_root}/pymdp"]
    sys.modules["pymdp"] = pkg
    ffi = _module("pymdp.ffi",
                  can_handle_fpi=lambda *a, **k: False,
                  can_handle=lambda *a, **k: False,
                  neg_efe_ffi_beneficial=lambda *a, **k: False)
    pkg.ffi = ffi
    loaded = {}
    for name in modules:
        spec = importlib.util.spec_from_file_location(f"pymdp.{name}", f"{ref_root}/pymdp/{name}.py")
        mod = importlib.util.module_from_spec(spec)
        sys.modules[f"pymdp.{name}"] = mod
        setattr(pkg, name, mod)
        spec.loader.exec_module(mod)
        loaded[name] = mod
    return types.SimpleNamespace(**loaded)
