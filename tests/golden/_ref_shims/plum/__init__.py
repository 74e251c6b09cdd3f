"""Minimal stand-in for the ``plum`` multiple-dispatch package.

ipie selects implementations with ``@plum.dispatch`` on type annotations.  The
real package is not installed in this container, so fixture generation imports
ipie with this shim on ``sys.path``.  Dispatch rule: the most recently
registered definition whose annotated parameters all pass ``isinstance`` wins.
Only used by ``tests/golden/make_golden.py``; nothing in the product imports it.
"""
import inspect
import typing

_registry = {}


def _resolve(ann, globs):
    if isinstance(ann, str):
        try:
            ann = eval(ann, globs)  # forward reference such as "SingleDet"
        except Exception:
            return None
    return ann


def _matches(value, ann, globs):
    ann = _resolve(ann, globs)
    if ann is None or ann is inspect.Parameter.empty or ann is typing.Any:
        return True
    if isinstance(ann, typing.TypeVar):
        return True
    origin = typing.get_origin(ann)
    if origin is typing.Union:
        return any(_matches(value, a, globs) for a in typing.get_args(ann))
    if origin is not None:
        ann = origin
    if ann is type(None):
        return value is None
    try:
        return isinstance(value, ann)
    except TypeError:
        return True


def _make_dispatcher(key):
    def dispatcher(*args, **kwargs):
        for fn, sig in reversed(_registry[key]):
            try:
                bound = sig.bind(*args, **kwargs)
            except TypeError:
                continue
            ok = True
            for name, val in bound.arguments.items():
                p = sig.parameters[name]
                if p.kind in (p.VAR_POSITIONAL, p.VAR_KEYWORD):
                    continue
                if not _matches(val, p.annotation, fn.__globals__):
                    ok = False
                    break
            if ok:
                return fn(*args, **kwargs)
        raise TypeError(f"no dispatch match for {key}")

    dispatcher.__name__ = key[1].split(".")[-1]
    return dispatcher


class _Dispatch:
    def __call__(self, fn):
        key = (fn.__module__, fn.__qualname__)
        _registry.setdefault(key, []).append((fn, inspect.signature(fn)))
        return _make_dispatcher(key)

    def abstract(self, fn):
        key = (fn.__module__, fn.__qualname__)
        _registry.setdefault(key, [])
        return _make_dispatcher(key)


dispatch = _Dispatch()
