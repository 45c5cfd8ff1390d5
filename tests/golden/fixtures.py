"""Flat npz (de)serialisation of nested dict/list fixtures (test infrastructure)."""
import json

import numpy


def _flatten(obj, prefix, out, meta):
    if isinstance(obj, dict):
        meta[prefix] = ["dict", sorted(obj.keys())]
        for k in obj:
            _flatten(obj[k], prefix + "/" + str(k), out, meta)
    elif isinstance(obj, (list, tuple)):
        meta[prefix] = ["list", len(obj)]
        for i, v in enumerate(obj):
            _flatten(v, prefix + "/" + str(i), out, meta)
    else:
        out[prefix] = numpy.asarray(obj)


def save(path, obj):
    out, meta = {}, {}
    _flatten(obj, "", out, meta)
    out["__meta__"] = numpy.array(json.dumps(meta))
    numpy.savez_compressed(path, **out)


def load(path):
    z = numpy.load(path, allow_pickle=False)
    meta = json.loads(str(z["__meta__"]))

    def build(prefix):
        m = meta.get(prefix)
        if m is None:
            a = z[prefix]
            return a.item() if a.ndim == 0 and a.dtype.kind in "iufb" else a
        if m[0] == "dict":
            return {k: build(prefix + "/" + k) for k in m[1]}
        return [build(prefix + "/" + str(i)) for i in range(m[1])]

    return build("")
