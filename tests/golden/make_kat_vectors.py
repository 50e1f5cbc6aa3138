"""Generate tests/golden/kat_vectors.json: known-answer vectors of the photon-walk functions.

Each case restates the inputs and the published expected value of one unit test of the
reference (stable/1.2/xmcml/xmcml_tests/*.cpp, CppUnit, tolerance `delta`; cited per case), and
records the value the reference's own code returns for the same inputs, computed here through the
reference build oracle/_ref/libxmcml_ref.so (base/ sources). The tests then check the oracle against
both: the published value within delta, the reference's value to the last bit.

Run from the repository root (needs oracle/_ref built from the reference sources):
    python tests/golden/make_kat_vectors.py
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import bind as B  # noqa: E402
from xmcml_b200 import structs as S  # noqa: E402

PI = 3.14159265358979323846
KT = "stable/1.2/xmcml/xmcml_tests/McmlKernelTestCase.cpp"
IT = "stable/1.2/xmcml/xmcml_tests/McmlIntersectionTestCase.cpp"
MT = "stable/1.2/xmcml/xmcml_tests/MCG59TestCase.cpp"

CASES = []


def case(kind, cite, args, expected, delta=1e-7):
    CASES.append({"kind": kind, "cite": cite, "args": args, "expected": expected, "delta": delta})


# --- MCG59 stream of seed 777, id 0, step 1 (first draws quoted in McmlKernelTestCase.cpp:14)
case("mcg59", KT + ":14", {"seed": 777, "id": 0, "step": 1, "n": 2}, [0.81700408, 0.41785875], 1e-8)
case("mcg59", MT + ":20-26", {"seed": 777, "id": 0, "step": 1, "n": 64}, None)
case("mcg59", MT + ":28-32", {"seed": 777, "id": 3, "step": 8, "n": 64}, None)
# --- specular reflectance (McmlKernelTestCase.cpp:37-115): layers (n0, n1, mua1, mus1, n2)
case("specular", KT + ":37-54", [1.0, 1.4, 1.0, 1.0, 1.0], 0.027777778)
case("specular", KT + ":56-73", [1.0, 2.0, 1.0, 1.0, 1.0], 1.0 / 9.0)
case("specular", KT + ":75-92", [1.0, 2.0, 0.0, 0.0, 3.0], 1.0 / 7.0)
case("specular", KT + ":94-111", [1.0, 1.0, 0.0, 0.0, 3.0], 0.25)
# --- HG cos(theta) with the first draw of the seed-777 stream (McmlKernelTestCase.cpp:737-769)
case("cosine_theta", KT + ":737-742", {"g": 0.5}, 0.925699)
case("cosine_theta", KT + ":744-749", {"g": 0.9}, 0.9974254)
case("cosine_theta", KT + ":751-756", {"g": 0.0}, 0.63400816)
# --- new direction, g = 0.5 (McmlKernelTestCase.cpp:775-832)
case("direction", KT + ":775-792", {"g": 0.5, "dir": [0.0, 0.0, 1.0]}, [-0.3289909967, 0.1866715735, 0.9256990049])
case("direction", KT + ":794-812", {"g": 0.5, "dir": [0.5, 0.5, 0.5], "normalize": True},
     [0.2681458221, 0.5321392932, 0.8030725936])
case("direction", KT + ":814-832", {"g": 0.5, "dir": [0.1, 0.2, 0.5], "normalize": True},
     [-0.132265401, 0.152879525, 0.979353722])
# --- transmit cosine (McmlKernelTestCase.cpp:838-907): (n_i, n_t, cos_i)
case("transmit_cos", KT + ":838-847", [1.1, 1.2, math.cos(PI / 4.0)], 0.7614861)
case("transmit_cos", KT + ":849-858", [1.0, 1.2, math.cos(PI / 4.0)], 0.8079466)
case("transmit_cos", KT + ":860-869", [1.1, 1.1, math.cos(PI / 4.0)], math.cos(PI / 4.0))
case("transmit_cos", KT + ":871-880", [1.1, 1.2, math.cos(0.00001)], math.cos(0.00001))
case("transmit_cos", KT + ":882-891", [1.1, 1.2, math.cos(PI / 1.99999)], 0.0)
case("transmit_cos", KT + ":893-902", [1.5, 1.0, math.cos(PI / 3.0)], 0.0)
# --- Fresnel reflectance (McmlKernelTestCase.cpp:914-977): (n_i, n_t, cos_i, cos_t)
case("fresnel", KT + ":914-923", [1.0, 1.2, math.cos(PI / 3.0), math.cos(PI / 4.0)], 0.0384758)
case("fresnel", KT + ":925-934", [1.0, 1.2, math.cos(PI / 3.0), math.cos(PI / 6.0)], 0.125)
case("fresnel", KT + ":936-945", [1.1, 1.1, math.cos(PI / 3.0), math.cos(PI / 6.0)], 0.0)
case("fresnel", KT + ":947-956", [1.1, 1.2, math.cos(0.0000001), math.cos(PI / 6.0)], 0.001890359)
case("fresnel", KT + ":958-967", [1.1, 1.2, math.cos(PI / 2.00000001), math.cos(PI / 6.0)], 1.0)
case("fresnel", KT + ":969-977", [1.1, 1.2, math.cos(PI / 3.0), math.cos(0.0)], 1.0)
# --- FindIntersectionLayer on a 4-layer topology (McmlKernelTestCase.cpp:984-1135)
TOPO = [[0, 2, 4], [0, 1, 3], [1, 2, 5], [3, 4, 5]]
case("find_layer", KT + ":984-1019", {"topology": TOPO, "surface": 1, "current": 1}, 2, 0)
case("find_layer", KT + ":1021-1056", {"topology": TOPO, "surface": 3, "current": 3}, 1, 0)
case("find_layer", KT + ":1058-1093", {"topology": TOPO, "surface": 2, "current": 2}, 0, 0)
case("find_layer", KT + ":1095-1130", {"topology": TOPO, "surface": 6, "current": 1}, -1, 0)
# --- refract / reflect (McmlKernelTestCase.cpp:1148-1240)
case("refract", KT + ":1148-1163", {"ni": 1.1, "nt": 1.2, "i": [1.0, -1.0, 0.0], "n": [0.0, 1.0, 0.0]},
     [0.648181216, -0.7614861201, 0.0])
case("refract", KT + ":1165-1180", {"ni": math.sqrt(3.0), "nt": 2 * math.sqrt(3.0), "i": [1.0, 1.0, 1.0], "n": [1.0, 0.0, 0.0]},
     [math.sqrt(10.0) / math.sqrt(12.0), 1.0 / math.sqrt(12.0), 1.0 / math.sqrt(12.0)])
case("reflect", KT + ":1186-1201", {"i": [1.0, -1.0, 0.0], "n": [0.0, -1.0, 0.0]}, [1 / math.sqrt(2.0), 1 / math.sqrt(2.0), 0.0])
case("reflect", KT + ":1203-1218", {"i": [0.0, -1.0, 0.0], "n": [1.0, 1.0, 0.0]}, [1.0, 0.0, 0.0])
case("reflect", KT + ":1220-1235", {"i": [0.0, -1.0, 0.0], "n": [1.0, 1.0, 1.0]}, [2 / 3.0, -1 / 3.0, 2 / 3.0])
# --- step size with the first draw (McmlKernelTestCase.cpp:1246-1272)
case("step_size", KT + ":1246-1258", {"mua": 20.0, "mus": 100.0}, 0.00168426)
case("step_size", KT + ":1260-1272", {"mua": 4.0, "mus": 5.0}, 0.0224568)
# --- dropped weight: photon weights after the drop (McmlKernelTestCase.cpp:1282-1360). The 1.2
# tests also assert absorption += 1/mus (an estimator that base/ replaced by += dw); only the
# weights are restated here, base's dw = w mua / (mua + mus) is checked against the reference build.
case("drop", KT + ":1282-1305", {"w": 0.8, "mua": 20.0, "mus": 200.0, "calls": 1}, 0.72727273)
case("drop", KT + ":1307-1330", {"w": 0.7, "mua": 10.0, "mus": 100.0, "calls": 1}, 0.63636364)
case("drop", KT + ":1332-1360", {"w": 1.0, "mua": 10.0, "mus": 90.0, "calls": 2}, 0.81)
# --- critical cosine (McmlKernelTestCase.cpp:1371-1398): layer indices into n = (1, 2, 1)
case("critical_cos", KT + ":1371-1383", {"n": [1.0, 2.0, 1.0], "cur": 1, "next": 2}, math.sqrt(3.0) / 2.0)
case("critical_cos", KT + ":1385-1397", {"n": [1.0, 2.0, 1.0], "cur": 0, "next": 1}, 0.0)
# --- area index (McmlKernelTestCase.cpp:463-731): corner, length, partitions, position
case("area_index", KT + ":463-488", {"corner": [0, 0, 0], "length": [1, 1, 1], "parts": [100, 100, 100], "p": [0.5, 0.5, 0.5]}, 505050, 0)
case("area_index", KT + ":490-515", {"corner": [0, 0, 0], "length": [1, 1, 1], "parts": [99, 99, 99], "p": [0.5, 0.5, 0.5]}, 485149, 0)
case("area_index", KT + ":517-542", {"corner": [0, 0, 0], "length": [1, 1, 1], "parts": [100, 100, 100], "p": [0.9999, 0.9999, 0.9999]}, 999999, 0)
case("area_index", KT + ":544-569", {"corner": [1, 1, 1], "length": [1, 1, 1], "parts": [100, 100, 100], "p": [1.5, 1.5, 1.5]}, 505050, 0)
case("area_index", KT + ":571-596", {"corner": [-1.5, -1.4, 0.3], "length": [2, 2, 2], "parts": [10, 20, 30], "p": [-0.9, 0.0, 0.5]}, 2223, 0)
case("area_index", KT + ":598-623", {"corner": [0, 0, 0], "length": [1, 1, 1], "parts": [3, 3, 3], "p": [0.5, 0.5, 0.5]}, 13, 0)
case("area_index", KT + ":625-650", {"corner": [1, 1, 1], "length": [1, 1, 1], "parts": [100, 100, 100], "p": [1.5, 1.5, 2.5]}, -1, 0)
case("area_index", KT + ":652-677", {"corner": [1, 1, 1], "length": [1, 1, 1], "parts": [100, 100, 100], "p": [-1.5, 1.5, 1.5]}, -1, 0)
case("area_index", KT + ":679-704", {"corner": [-100, -100, -100], "length": [200, 200, 200], "parts": [10, 10, 10], "p": [-104.5, 1.5, 1.5]}, -1, 0)
case("area_index", KT + ":706-731", {"corner": [0, 0, 0], "length": [1, 1, 1], "parts": [100, 100, 100], "p": [1.0, 1.0, 1.0]}, -1, 0)
# --- ray-triangle distance (McmlIntersectionTestCase.cpp:19-90); None = miss (>= MAX_DISTANCE)
TRI1 = [[2.0, -1.0, -1.0], [2.0, 1.0, -1.0], [2.0, 0.0, 2.0]]
case("triangle", IT + ":19-28", {"o": [0, 0, 0], "d": [1, 0, 0], "tri": TRI1}, 2.0)
case("triangle", IT + ":29-38", {"o": [0, 0, 0], "d": [1, 0, 0], "tri": [[0, -1, -1], [0, 1, -1], [2.25, 0, 1]]}, 1.125)
case("triangle", IT + ":39-48", {"o": [0, 0, 0], "d": [-1, 0, 0], "tri": TRI1}, -2.0)
case("triangle", IT + ":49-58", {"o": [0, 0, 0], "d": [1, 0, 0], "tri": [[0, -1, -1], [0, 1, -1], [0, 0, 1]]}, 0.0)
case("triangle", IT + ":59-68", {"o": [0, 0, 0], "d": [1, 0, 0], "tri": [[1, 0, 5], [0, 1, 5], [0, 0, 5]]}, None)
case("triangle", IT + ":69-78", {"o": [0, 3, -1], "d": [1, 0, 0], "tri": TRI1}, None)
case("triangle", IT + ":79-88", {"o": [0, 1, 0], "d": [1, 0, 0], "tri": TRI1}, None)


def _arr(v):
    return (C.c_double * len(v))(*[float(x) for x in v])


def reference_value(c):
    """The reference's own code on the case inputs (oracle/_ref/libxmcml_ref.so)."""
    L = B.ref()
    k, a = c["kind"], c["args"]
    if k == "mcg59":
        g = S.MCG59()
        L.ref_init_mcg59(C.byref(g), a["seed"], a["id"], a["step"])
        return [L.ref_next_mcg59(C.byref(g)) for _ in range(a["n"])]
    if k == "specular":
        lay = (S.LayerInfo * 3)()
        lay[0].refractiveIndex, lay[1].refractiveIndex, lay[1].absorptionCoefficient = a[0], a[1], a[2]
        lay[1].scatteringCoefficient, lay[2].refractiveIndex = a[3], a[4]
        return L.ref_specular(lay)
    if k in ("cosine_theta", "direction", "step_size"):
        g = S.MCG59()
        L.ref_init_mcg59(C.byref(g), 777, 0, 1)
        if k == "cosine_theta":
            return L.ref_cosine_theta(a["g"], C.byref(g))
        if k == "step_size":
            return L.ref_step_size(a["mua"], a["mus"], C.byref(g))
        d = list(a["dir"])
        if a.get("normalize"):
            n = math.sqrt(sum(x * x for x in d))
            d = [x / n for x in d]
        out = (C.c_double * 3)()
        L.ref_new_direction(_arr(d), a["g"], C.byref(g), out)
        return list(out)
    if k == "transmit_cos":
        return L.ref_transmit_cos(*a)
    if k == "fresnel":
        return L.ref_fresnel(*a)
    if k == "find_layer":
        info, keep = topology_input(a["topology"])
        return L.ref_find_layer(C.byref(info), a["surface"], a["current"])
    if k == "refract":
        out = (C.c_double * 3)()
        L.ref_refract(a["ni"], a["nt"], _arr(a["i"]), _arr(a["n"]), out)
        return list(out)
    if k == "reflect":
        out = (C.c_double * 3)()
        L.ref_reflect(_arr(a["i"]), _arr(a["n"]), out)
        return list(out)
    if k == "drop":
        w = a["w"]
        total = 0.0
        for _ in range(a["calls"]):
            dw = C.c_double()
            w = L.ref_drop(w, a["mua"], a["mus"], C.byref(dw))
            total += dw.value
        return [w, total]
    if k == "critical_cos":
        lay = (S.LayerInfo * 3)()
        for i, n in enumerate(a["n"]):
            lay[i].refractiveIndex = n
        return L.ref_critical_cos(lay, a["cur"], a["next"])
    if k == "area_index":
        return L.ref_area_index(_arr(a["p"]), C.byref(area(a)))
    if k == "triangle":
        t = a["tri"]
        v = L.ref_triangle(_arr(a["o"]), _arr(a["d"]), _arr(t[0]), _arr(t[1]), _arr(t[2]))
        return None if v >= 1e256 else v
    raise ValueError(k)


def area(a):
    ar = S.Area()
    ar.corner = S.double3(*[float(x) for x in a["corner"]])
    ar.length = S.double3(*[float(x) for x in a["length"]])
    ar.partitionNumber = S.int3(*a["parts"])
    return ar


def topology_input(topo):
    info = S.InputInfo()
    lay = (S.LayerInfo * len(topo))()
    keep = []
    for i, ids in enumerate(topo):
        arr = (C.c_int * len(ids))(*ids)
        keep.append(arr)
        lay[i].surfaceId = C.cast(arr, C.POINTER(C.c_int))
        lay[i].numberOfSurfaces = len(ids)
    info.layerInfo = C.cast(lay, C.POINTER(S.LayerInfo))
    info.numberOfLayers = len(topo)
    keep.append(lay)
    return info, keep


def main():
    out = []
    for c in CASES:
        c = dict(c)
        c["reference"] = reference_value(c)
        out.append(c)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kat_vectors.json")
    with open(path, "w") as f:
        json.dump({"generator": "tests/golden/make_kat_vectors.py", "cases": out}, f, indent=1)
    print(f"wrote {len(out)} cases to {path}")


if __name__ == "__main__":
    main()
