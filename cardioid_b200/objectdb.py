"""Reader and writer for Cardioid's object-database text format.

The reference keeps every input in ``object.data`` files of objects

    name CLASS { key = value value ...; key = value unit; }

parsed by simUtil/src/object.c (``object_compilefile``) and queried with
``objectGet(obj, key, value, default, unit)`` (simUtil/src/object_cc.cc).
This module reads the same syntax (``//`` and ``#`` line comments, ``/* */``
blocks) so a user's REACTION / FIT / FUNCTION / STIMULUS / DIFFUSION objects
drive the B200 engine unchanged.  Units: Cardioid's internal and external
units are the same (mm, ms, mV, mS, uF; elec/cardioid.cc:43-63, 84-85), so a
value given with its natural unit word is taken as is; a unit word is kept
for reference only.
"""
import re

_COMMENT = re.compile(r"//[^\n]*|#[^\n]*|/\*.*?\*/", re.S)
_OBJECT = re.compile(r"([A-Za-z_][\w.\-]*)\s+([A-Za-z_]\w*)\s*\{(.*?)\}", re.S)


class ObjectDB:
    """A set of objects keyed by (name, CLASS).  Later definitions of the same
    object merge key by key, as object_compilefile does when an object is
    declared twice (e.g. ``tt06 REACTION { fit=tt06_fit; }`` in a fit file)."""

    def __init__(self):
        self.objects = {}
        self.order = []

    def compile(self, text):
        text = _COMMENT.sub("", text)
        for name, cls, body in _OBJECT.findall(text):
            key = (name, cls.upper())
            obj = self.objects.get(key)
            if obj is None:
                obj = {}
                self.objects[key] = obj
                self.order.append(key)
            for stmt in body.split(";"):
                if "=" not in stmt:
                    continue
                k, v = stmt.split("=", 1)
                k = k.strip()
                if k:
                    obj[k] = v.split()
        return self

    def compile_file(self, path):
        with open(path) as f:
            return self.compile(f.read())

    def find(self, name, cls):
        obj = self.objects.get((name, cls.upper()))
        if obj is None:
            raise KeyError("object %s %s not found" % (name, cls))
        return obj

    def exists(self, name, cls):
        return (name, cls.upper()) in self.objects

    def names(self, cls):
        return [n for (n, c) in self.order if c == cls.upper()]


def get_str(obj, key, default=None):
    v = obj.get(key)
    if not v:
        return default
    return v[0]


def get_list(obj, key):
    return list(obj.get(key, []))


def get_float(obj, key, default=None):
    """objectGet for a scalar: the first word, parsed as a number.  A trailing
    unit word is accepted and ignored (internal units == external units)."""
    v = obj.get(key)
    if not v:
        if default is None:
            return None
        return float(default)
    return float(v[0])


def get_floats(obj, key):
    return [float(x) for x in obj.get(key, [])]


def format_float(x):
    """Shortest text that reads back to the same double (the reference writes
    fits with precision 16, BetterTT06.cc:159; 17 significant digits keep
    every double exact)."""
    r = repr(float(x))
    return r
