"""A numpy-backed stand-in for the parts of JAX that WRF-JAX's RRTMG path uses.

This module exists only to generate golden fixtures: it lets the reference's
own ``rrtmg_lwrad_wrf_columns`` / ``rrtmg_swrad_wrf_columns`` (and their inner
functions) execute in a container that has numpy but no jax/jaxlib, so that the
fixtures under ``tests/golden/`` are outputs of the reference's code rather
than of this project's restatement.

Semantics kept from JAX with ``jax_enable_x64=True``:

* every jnp/lax operation is evaluated eagerly by numpy with the same dtypes
  (float32 arithmetic is IEEE binary32, float64 binary64, integers wrap);
* Python scalars stay weakly typed (numpy >= 2 follows NEP 50, which matches
  JAX's weak-type promotion for scalars);
* ``x.at[idx].set/add/...`` return updated copies;
* ``lax.scan`` / ``fori_loop`` / ``vmap`` run as Python loops;
* ``jax.config.jax_disable_jit`` reports True so that the reference takes its
  plain ``lax.scan`` branch instead of its Pallas/Triton one;
* custom JVP / batching rules are accepted and ignored (no differentiation).

Nothing in the product imports this file.
"""

from __future__ import annotations

import ctypes
import ctypes.util
import sys
import types

import numpy as np

_LIBM = ctypes.CDLL(ctypes.util.find_library("m"))
_LIBM.expf.restype = ctypes.c_float
_LIBM.expf.argtypes = [ctypes.c_float]


# ----------------------------------------------------------------------------
# array type with JAX's functional ``.at`` updates
# ----------------------------------------------------------------------------
class Arr(np.ndarray):
    """ndarray subclass carrying JAX's ``.at[...]`` update syntax."""

    @property
    def at(self):
        return _At(self)

    def block_until_ready(self):
        return self

    def __hash__(self):  # JAX arrays are unhashable too, but lru_cache keys never hold them
        raise TypeError("unhashable array")

    def __getitem__(self, idx):
        # JAX gathers clamp out-of-range integer-array indices instead of raising.
        return super().__getitem__(_clamp_index(idx, self.shape))

    def __pow__(self, other):
        # ``x ** n`` with a Python int is lax.integer_pow (repeated squaring).
        if isinstance(other, int) and not isinstance(other, bool):
            return _integer_pow(self.view(np.ndarray), other)
        return super().__pow__(other)


def _clamp_index(idx, shape):
    if not isinstance(idx, tuple):
        idx = (idx,)
    n_consumed = sum(1 for i in idx if i is not None and i is not Ellipsis and not (
        isinstance(i, np.ndarray) and i.dtype == bool))
    out, axis = [], 0
    for i in idx:
        if i is Ellipsis:
            axis += len(shape) - n_consumed
            out.append(i)
            continue
        if i is None:
            out.append(i)
            continue
        if isinstance(i, np.ndarray) and i.dtype != bool and np.issubdtype(i.dtype, np.integer):
            n = shape[axis]
            j = np.asarray(i).view(np.ndarray).astype(np.int64)
            j = np.where(j < 0, j + n, j)
            out.append(np.clip(j, 0, n - 1))
        else:
            out.append(i.view(np.ndarray) if isinstance(i, Arr) else i)
        axis += 1
    return tuple(out)


class _At:
    def __init__(self, base):
        self._base = base

    def __getitem__(self, idx):
        return _AtRef(self._base, idx)


class _AtRef:
    def __init__(self, base, idx):
        self._base, self._idx = base, _fix_index(idx)

    def _copy(self):
        return np.array(self._base, copy=True)

    def set(self, value, **_):
        out = self._copy()
        out[self._idx] = np.asarray(value)
        return out.view(Arr)

    def add(self, value, **_):
        out = self._copy()
        np.add.at(out, self._idx, np.asarray(value, dtype=out.dtype))
        return out.view(Arr)

    def multiply(self, value, **_):
        out = self._copy()
        np.multiply.at(out, self._idx, np.asarray(value, dtype=out.dtype))
        return out.view(Arr)

    def min(self, value, **_):
        out = self._copy()
        np.minimum.at(out, self._idx, np.asarray(value, dtype=out.dtype))
        return out.view(Arr)

    def max(self, value, **_):
        out = self._copy()
        np.maximum.at(out, self._idx, np.asarray(value, dtype=out.dtype))
        return out.view(Arr)

    def get(self, **_):
        return wrap(np.asarray(self._base)[self._idx])


def _fix_index(idx):
    if isinstance(idx, tuple):
        return tuple(_fix_index(i) for i in idx)
    if isinstance(idx, np.ndarray) and not isinstance(idx, (np.bool_,)) and idx.dtype != bool:
        return np.asarray(idx)
    return idx


def wrap(value):
    """Convert numpy results into ``Arr`` (recursively through tuples/lists)."""
    if isinstance(value, Arr):
        return value
    if isinstance(value, np.ndarray):
        return value.view(Arr)
    if isinstance(value, np.generic):
        return np.asarray(value).view(Arr)
    if isinstance(value, tuple) and not hasattr(value, "_fields"):
        return tuple(wrap(v) for v in value)
    if isinstance(value, list):
        return [wrap(v) for v in value]
    return value


def _plain(value):
    if isinstance(value, Arr):
        return value.view(np.ndarray)
    return value


# ----------------------------------------------------------------------------
# pytrees
# ----------------------------------------------------------------------------
def _is_leaf(x):
    return not isinstance(x, (tuple, list, dict)) or (x is None)


def tree_flatten(tree):
    leaves = []

    def rec(x):
        if x is None:
            return ("none",)
        if isinstance(x, tuple) and hasattr(x, "_fields"):
            return ("nt", type(x), tuple(rec(v) for v in x))
        if isinstance(x, tuple):
            return ("tuple", tuple(rec(v) for v in x))
        if isinstance(x, list):
            return ("list", tuple(rec(v) for v in x))
        if isinstance(x, dict):
            keys = sorted(x)
            return ("dict", tuple(keys), tuple(rec(x[k]) for k in keys))
        leaves.append(x)
        return ("leaf",)

    return leaves, rec(tree)


def tree_unflatten(treedef, leaves):
    it = iter(leaves)

    def rec(d):
        kind = d[0]
        if kind == "none":
            return None
        if kind == "leaf":
            return next(it)
        if kind == "nt":
            return d[1](*(rec(c) for c in d[2]))
        if kind == "tuple":
            return tuple(rec(c) for c in d[1])
        if kind == "list":
            return [rec(c) for c in d[1]]
        if kind == "dict":
            return {k: rec(c) for k, c in zip(d[1], d[2])}
        raise AssertionError(kind)

    return rec(treedef)


def tree_map(f, tree, *rest, is_leaf=None):
    leaves, treedef = tree_flatten(tree)
    others = [tree_flatten(r)[0] for r in rest]
    return tree_unflatten(treedef, [f(*xs) for xs in zip(leaves, *others)])


def tree_leaves(tree, is_leaf=None):
    return tree_flatten(tree)[0]


def tree_structure(tree):
    return _TreeDef(tree_flatten(tree)[1])


class _TreeDef:
    def __init__(self, d):
        self.d = d

    def __eq__(self, other):
        return isinstance(other, _TreeDef) and self.d == other.d

    def __ne__(self, other):
        return not self == other


def _broadcast_prefix(prefix, tree):
    """Expand a pytree prefix (e.g. vmap in_axes) to the full structure of tree."""
    if prefix is None or isinstance(prefix, int):
        leaves, treedef = tree_flatten(tree)
        return tree_unflatten(treedef, [prefix] * len(leaves)), leaves
    if isinstance(tree, tuple) and hasattr(tree, "_fields"):
        parts = [_broadcast_prefix(p, t) for p, t in zip(prefix, tree)]
        return type(tree)(*(p[0] for p in parts)), [l for p in parts for l in p[1]]
    if isinstance(tree, (tuple, list)):
        parts = [_broadcast_prefix(p, t) for p, t in zip(prefix, tree)]
        return type(tree)(p[0] for p in parts), [l for p in parts for l in p[1]]
    if isinstance(tree, dict):
        parts = {k: _broadcast_prefix(prefix[k], tree[k]) for k in tree}
        return {k: v[0] for k, v in parts.items()}, [l for k in sorted(tree) for l in parts[k][1]]
    raise TypeError(f"cannot broadcast prefix {prefix!r}")


# ----------------------------------------------------------------------------
# transformations
# ----------------------------------------------------------------------------
def vmap(fun, in_axes=0, out_axes=0, **_):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        full_axes = []
        size = None
        for arg, ax in zip(args, axes):
            expanded, _ = _broadcast_prefix(ax, arg)
            full_axes.append(expanded)
            for leaf, lax_ in zip(tree_leaves(arg), tree_flatten(expanded)[0] if not isinstance(expanded, int) and expanded is not None else [expanded] * len(tree_leaves(arg))):
                if lax_ is not None:
                    size = np.shape(leaf)[lax_]
        if size is None:
            raise ValueError("vmap needs at least one mapped argument")
        outs = []
        for i in range(size):
            call_args = []
            for arg, ax in zip(args, full_axes):
                leaves, treedef = tree_flatten(arg)
                ax_leaves = [ax] * len(leaves) if (ax is None or isinstance(ax, int)) else _axes_leaves(ax, len(leaves))
                sliced = [wrap(np.take(np.asarray(l), i, axis=a)) if a is not None else l for l, a in zip(leaves, ax_leaves)]
                call_args.append(tree_unflatten(treedef, sliced))
            outs.append(fun(*call_args))
        return tree_map(lambda *xs: wrap(np.stack([np.asarray(x) for x in xs], axis=out_axes)), outs[0], *outs[1:])

    return mapped


def _axes_leaves(ax_tree, n):
    # Leaves of an expanded axes tree; None entries are leaves here.
    out = []

    def rec(x):
        if x is None or isinstance(x, int):
            out.append(x)
        elif isinstance(x, dict):
            for k in sorted(x):
                rec(x[k])
        else:
            for v in x:
                rec(v)

    rec(ax_tree)
    assert len(out) == n, (len(out), n)
    return out


def jit(fun=None, **_):
    if fun is None:
        return lambda f: f
    return fun


class custom_jvp:
    def __init__(self, fun, nondiff_argnums=()):
        self.fun = fun
        self.__wrapped__ = fun
        self.__name__ = getattr(fun, "__name__", "custom_jvp")

    def defjvp(self, rule, **_):
        return rule

    def defjvps(self, *rules):
        return None

    def __call__(self, *args, **kwargs):
        return self.fun(*args, **kwargs)


class custom_vmap:
    def __init__(self, fun):
        self.fun = fun

    def def_vmap(self, rule):
        return rule

    def __call__(self, *args, **kwargs):
        return self.fun(*args, **kwargs)


class ShapeDtypeStruct:
    def __init__(self, shape, dtype):
        self.shape = tuple(shape)
        self.dtype = np.dtype(dtype)
        self.ndim = len(self.shape)
        self.size = int(np.prod(self.shape)) if self.shape else 1


def eval_shape(fun, *args, **kwargs):
    def concrete(x):
        if isinstance(x, ShapeDtypeStruct):
            return wrap(np.zeros(x.shape, x.dtype))
        return x

    out = fun(*tree_map(concrete, args), **kwargs)
    return tree_map(lambda x: ShapeDtypeStruct(np.shape(x), np.asarray(x).dtype), out)


# ----------------------------------------------------------------------------
# jax.numpy
# ----------------------------------------------------------------------------
def _make_jnp():
    jnp = types.ModuleType("jax.numpy")
    for name in ("float16", "float32", "float64", "int8", "int16", "int32", "int64",
                 "uint8", "uint16", "uint32", "uint64", "bool_", "complex64",
                 "pi", "inf", "nan", "e", "newaxis", "dtype", "ndarray", "iinfo", "finfo",
                 "integer", "floating", "number", "signedinteger", "unsignedinteger"):
        setattr(jnp, name, getattr(np, name))
    jnp.bfloat16 = np.float32

    def asarray(x, dtype=None, **_):
        if dtype is None and isinstance(x, (bool, int, float)) and not isinstance(x, np.generic):
            # Keep Python scalars weakly typed, as JAX does.
            return x
        if dtype is None and isinstance(x, (list, tuple)) and x and all(
                isinstance(v, float) and not isinstance(v, np.generic) for v in x):
            return wrap(np.asarray(x, dtype=np.float64))
        return wrap(np.asarray(_plain(x), dtype=dtype))

    jnp.asarray = asarray
    jnp.array = lambda x, dtype=None, copy=True, **k: wrap(np.array(_plain(x) if not isinstance(x, (int, float)) or dtype is not None else x, dtype=dtype, copy=copy))

    def _wrapfn(f):
        def g(*args, **kwargs):
            return wrap(f(*[_plain(a) for a in args], **kwargs))
        g.__name__ = getattr(f, "__name__", "fn")
        return g

    def where(cond, x=None, y=None):
        if x is None:
            return wrap(np.where(cond))
        return wrap(np.where(_plain(cond), _plain(x), _plain(y)))

    jnp.where = where

    def clip(a, a_min=None, a_max=None, *, min=None, max=None):
        lo = a_min if a_min is not None else min
        hi = a_max if a_max is not None else max
        return wrap(np.clip(_plain(a), lo, hi))

    jnp.clip = clip

    def take(a, indices, axis=None, mode=None, **_):
        arr = np.asarray(_plain(a))
        idx = np.asarray(_plain(indices))
        n = arr.shape[axis] if axis is not None else arr.size
        idx = np.clip(idx, -n, n - 1)  # JAX clamps out-of-range gathers
        return wrap(np.take(arr, idx, axis=axis))

    jnp.take = take

    def power(x, y):
        xp = _plain(x)
        if isinstance(y, int) and not isinstance(y, bool):
            return _integer_pow(xp, y)
        return wrap(np.power(xp, _plain(y)))

    jnp.power = power

    def full(shape, fill_value, dtype=None):
        if dtype is None:
            dtype = np.asarray(_plain(fill_value)).dtype
        return wrap(np.full(shape, _plain(fill_value), dtype=dtype))

    jnp.full = full

    class _Reducer:
        def __init__(self, ufunc):
            self.ufunc = ufunc

        def __call__(self, *args, **kwargs):
            return wrap(self.ufunc(*[_plain(a) for a in args], **kwargs))

        def reduce(self, a, axis=0, **kwargs):
            return wrap(self.ufunc.reduce(_plain(a), axis=axis, **kwargs))

    for name in ("bitwise_xor", "bitwise_and", "bitwise_or", "add", "multiply",
                 "maximum", "minimum", "logical_and", "logical_or"):
        setattr(jnp, name, _Reducer(getattr(np, name)))

    def max_(a, axis=None, initial=None, **kwargs):
        if initial is not None:
            kwargs["initial"] = initial
        return wrap(np.max(_plain(a), axis=axis, **kwargs))

    jnp.max = max_
    jnp.amax = max_

    def exp(x):
        arr = np.asarray(_plain(x))
        if arr.dtype == np.float32:
            # XLA's binary32 exp is not available here; use glibc expf, the
            # libm the reference emulates everywhere else on this path.
            flat = arr.reshape(-1)
            out = np.fromiter((_LIBM.expf(float(v)) for v in flat), dtype=np.float32, count=flat.size)
            return wrap(out.reshape(arr.shape))
        return wrap(np.exp(arr))

    jnp.exp = exp

    def _getattr(name):
        f = getattr(np, name)
        if callable(f):
            return _wrapfn(f)
        return f

    jnp.__getattr__ = _getattr
    return jnp


def _integer_pow(x, y):
    """lax.integer_pow: binary exponentiation in the operand's dtype."""
    x = np.asarray(x)
    if y == 0:
        return wrap(np.ones_like(x))
    is_reciprocal = y < 0
    y = abs(y)
    acc = None
    base = x
    while y:
        if y & 1:
            acc = base if acc is None else (acc * base).astype(x.dtype)
        y >>= 1
        if y:
            base = (base * base).astype(x.dtype)
    if is_reciprocal:
        acc = (np.asarray(1, dtype=x.dtype) / acc).astype(x.dtype)
    return wrap(acc)


# ----------------------------------------------------------------------------
# jax.lax
# ----------------------------------------------------------------------------
def _make_lax():
    lax = types.ModuleType("jax.lax")

    def scan(f, init, xs=None, length=None, reverse=False, unroll=1, **_):
        xs_leaves, xs_def = tree_flatten(xs)
        n = length if length is not None else np.shape(xs_leaves[0])[0]
        carry = init
        ys = [None] * n
        order = range(n - 1, -1, -1) if reverse else range(n)
        for i in order:
            x = tree_unflatten(xs_def, [wrap(np.asarray(l)[i]) for l in xs_leaves])
            carry, y = f(carry, x)
            ys[i] = y
        if n == 0:
            return carry, None
        if ys[0] is None:
            return carry, None
        stacked = tree_map(lambda *vals: wrap(np.stack([np.asarray(v) for v in vals])), ys[0], *ys[1:])
        return carry, stacked

    lax.scan = scan

    def fori_loop(lower, upper, body, init, **_):
        val = init
        for i in range(int(lower), int(upper)):
            val = body(np.int32(i), val)
        return val

    lax.fori_loop = fori_loop

    def cond(pred, true_fun, false_fun, *operands, **_):
        return true_fun(*operands) if bool(np.asarray(pred)) else false_fun(*operands)

    lax.cond = cond

    def platform_dependent(*args, **branches):
        fn = branches.get("cpu") or branches.get("default")
        return fn(*args)

    lax.platform_dependent = platform_dependent

    def dynamic_update_slice(operand, update, start_indices):
        # JAX clamps the start so that the update fits inside the operand
        out = np.array(_plain(operand), copy=True)
        upd = np.asarray(_plain(update))
        starts = [min(max(int(s), 0), out.shape[d] - upd.shape[d]) for d, s in enumerate(start_indices)]
        out[tuple(slice(s, s + n) for s, n in zip(starts, upd.shape))] = upd
        return wrap(out)

    lax.dynamic_update_slice = dynamic_update_slice
    lax.optimization_barrier = lambda x: x

    def bitcast_convert_type(x, new_dtype):
        arr = np.asarray(_plain(x))
        new_dtype = np.dtype(new_dtype)
        if arr.dtype.itemsize != new_dtype.itemsize:
            raise NotImplementedError("size-changing bitcast")
        return wrap(arr.view(new_dtype))

    lax.bitcast_convert_type = bitcast_convert_type
    lax.add = lambda a, b: wrap(np.add(_plain(a), _plain(b)))
    lax.sub = lambda a, b: wrap(np.subtract(_plain(a), _plain(b)))
    lax.mul = lambda a, b: wrap(np.multiply(_plain(a), _plain(b)))

    def div(a, b):
        a, b = np.asarray(_plain(a)), np.asarray(_plain(b))
        if np.issubdtype(a.dtype, np.integer):
            q = np.abs(a) // np.abs(b)
            return wrap((np.sign(a) * np.sign(b) * q).astype(a.dtype))
        return wrap(np.divide(a, b))

    lax.div = div
    lax.bitwise_xor = lambda a, b: wrap(np.bitwise_xor(_plain(a), _plain(b)))
    lax.bitwise_and = lambda a, b: wrap(np.bitwise_and(_plain(a), _plain(b)))
    lax.shift_right_arithmetic = lambda a, b: wrap(np.right_shift(_plain(a), _plain(b)))
    lax.shift_right_logical = lambda a, b: wrap(np.right_shift(_plain(a), _plain(b)))
    lax.shift_left = lambda a, b: wrap(np.left_shift(_plain(a), _plain(b)))
    lax.integer_pow = lambda x, y: _integer_pow(_plain(x), y)

    def reduce_precision(x, exponent_bits, mantissa_bits):
        if (exponent_bits, mantissa_bits) == (8, 23):
            return wrap(np.asarray(_plain(x)).astype(np.float32).astype(np.asarray(_plain(x)).dtype))
        raise NotImplementedError

    lax.reduce_precision = reduce_precision
    return lax


# ----------------------------------------------------------------------------
# jax._src pieces used by wrf_jax.core.real_arithmetic
# ----------------------------------------------------------------------------
class _Lowered:
    def __init__(self, fun):
        self.fun = fun

    def __call__(self, ctx, *args, **kwargs):
        return self.fun(*args, **kwargs)


class Primitive:
    def __init__(self, name):
        self.name = name
        self._impl = None

    def def_impl(self, f):
        return f

    def def_abstract_eval(self, f):
        return f

    def bind(self, *args, **params):
        if self._impl is None:
            raise NotImplementedError(self.name)
        return self._impl(*args, **params)


def _register_lowering(prim, rule, platform=None):
    if isinstance(rule, _Lowered):
        prim._impl = rule.fun
    else:
        prim._impl = lambda *a, **k: rule(None, *a, **k)


def _noop(*a, **k):
    return None


def install() -> None:
    """Register the stand-in modules under the ``jax`` names."""
    jax = types.ModuleType("jax")
    jnp = _make_jnp()
    lax = _make_lax()
    jax.numpy = jnp
    jax.lax = lax

    class _Config:
        x64_enabled = True
        jax_enable_x64 = True
        jax_disable_jit = True

        def update(self, *_a, **_k):
            return None

    jax.config = _Config()
    jax.jit = jit
    jax.vmap = vmap
    jax.custom_jvp = custom_jvp
    jax.ShapeDtypeStruct = ShapeDtypeStruct
    jax.eval_shape = eval_shape
    jax.Array = Arr
    jax.device_put = lambda x, *a, **k: x
    jax.block_until_ready = lambda x: x

    tree = types.ModuleType("jax.tree")
    tree.map = tree_map
    tree.leaves = tree_leaves
    tree.structure = tree_structure
    jax.tree = tree
    tree_util = types.ModuleType("jax.tree_util")
    tree_util.tree_map = tree_map
    tree_util.tree_leaves = tree_leaves
    tree_util.tree_structure = tree_structure
    tree_util.tree_flatten = tree_flatten
    jax.tree_util = tree_util

    debug = types.ModuleType("jax.debug")
    debug.callback = lambda f, *a, **k: f(*a, **k)
    jax.debug = debug

    custom_batching = types.ModuleType("jax.custom_batching")
    custom_batching.custom_vmap = custom_vmap
    jax.custom_batching = custom_batching

    src = types.ModuleType("jax._src")
    core = types.ModuleType("jax._src.core")
    core.Primitive = Primitive
    dispatch = types.ModuleType("jax._src.dispatch")
    dispatch.apply_primitive = _noop
    interpreters = types.ModuleType("jax._src.interpreters")
    ad = types.ModuleType("jax._src.interpreters.ad")
    for name in ("defjvp", "deflinear", "deflinear2", "defjvp_zero"):
        setattr(ad, name, _noop)
    batching = types.ModuleType("jax._src.interpreters.batching")
    batching.defbroadcasting = _noop
    batching.defvectorized = _noop
    mlir = types.ModuleType("jax._src.interpreters.mlir")
    mlir.register_lowering = _register_lowering
    mlir.lower_fun = lambda fun, multiple_results=False: _Lowered(fun)
    src.core, src.dispatch, src.interpreters = core, dispatch, interpreters
    interpreters.ad, interpreters.batching, interpreters.mlir = ad, batching, mlir
    jax._src = src

    for name, mod in {
        "jax": jax, "jax.numpy": jnp, "jax.lax": lax, "jax.tree": tree,
        "jax.tree_util": tree_util, "jax.debug": debug,
        "jax.custom_batching": custom_batching, "jax._src": src,
        "jax._src.core": core, "jax._src.dispatch": dispatch,
        "jax._src.interpreters": interpreters,
        "jax._src.interpreters.ad": ad, "jax._src.interpreters.batching": batching,
        "jax._src.interpreters.mlir": mlir,
    }.items():
        sys.modules[name] = mod
