"""The seeded boards (pcbroute_b200/dsngen.py) against the configurations they stand for.

Each board is parsed back from its Specctra text (the subset of the grammar pcbroute reads, src/dsn.cpp:75-384) and
checked for what the router and the timings depend on: the signal nets and two-pin connections of the
configuration (a net of k pins makes k - 1 connections), the multi-pin share and fan-out, the copper layers, the
plane nets, every pin reference naming a placed part's pad, no pad in two nets, parts inside the board outline and
not overlapping, and the same text for the same seed. CPU only.
"""
import re

import pytest

from pcbroute_b200 import dsngen


def _parse(text):
    layers = re.findall(r"\(layer (\S+) \(type signal\)\)", text)
    bx = [int(v) for v in re.search(r"\(boundary \(path pcb 0 ([^)]*)\)\)", text).group(1).split()]
    xs, ys = bx[0::2], bx[1::2]
    images = {}
    for m in re.finditer(r"\(image (\S+) ((?:\(pin [^)]*\) ?)+)\)", text):
        images[m.group(1)] = {p[1]: (int(p[2]), int(p[3])) for p in
                              (x.split() for x in re.findall(r"\(pin ([^)]*)\)", m.group(2)))}
    parts = {}
    for m in re.finditer(r"\(component (\S+) ((?:\(place [^)]*\) ?)+)\)", text):
        for p in re.findall(r"\(place ([^)]*)\)", m.group(2)):
            ref, x, y, side, rot = p.split()
            parts[ref] = (m.group(1), int(x), int(y), int(rot))
    nets = {m.group(1): m.group(2).split() for m in re.finditer(r"\(net (\S+) \(pins ([^)]*)\)\)", text)}
    planes = dict(re.findall(r"\(plane (\S+) \(polygon (\S+)", text))
    classes = {}
    for m in re.finditer(r"\(class (\S+) ([^(]*)\(circuit", text):
        for n in m.group(2).split():
            classes[n] = m.group(1)
    return dict(layers=layers, box=(min(xs), min(ys), max(xs), max(ys)), images=images, parts=parts, nets=nets,
                planes=planes, classes=classes)


@pytest.mark.parametrize("name", ["t1", "t2", "c1", "c2", "c4", "c5"])
def test_board_matches_its_configuration(name):
    cfg = dsngen.CONFIGS[name]
    b = _parse(dsngen.generate(name, 1))
    assert b["layers"] == cfg.layers
    signal = {n: p for n, p in b["nets"].items() if n not in b["planes"]}
    assert len(signal) == cfg.nets
    assert sum(len(p) - 1 for p in signal.values()) == cfg.connections
    assert all(len(p) >= 2 for p in signal.values())
    multi = [len(p) for p in signal.values() if len(p) > 2]
    if cfg.multipin_frac == 0:
        assert not multi
    else:
        assert all(cfg.fanout[0] <= k <= cfg.fanout[1] for k in multi), (min(multi), max(multi))
        assert abs(len(multi) / cfg.nets - cfg.multipin_frac) <= 0.1, len(multi) / cfg.nets
    # planes: one net per plane layer named by the configuration, with pins of its own
    assert sorted(b["planes"].items()) == sorted(cfg.planes)
    for net in b["planes"]:
        assert len(b["nets"].get(net, [])) >= 2
    # every pin reference is a pad of a placed part, and no pad belongs to two nets
    seen = set()
    for pins in b["nets"].values():
        for ref in pins:
            part, pin = ref.rsplit("-", 1)
            assert part in b["parts"], ref
            assert pin in b["images"][b["parts"][part][0]], ref
            assert ref not in seen, ref
            seen.add(ref)
    # the parts the configuration names are all there (pin-bearing parts may have been added)
    count = {}
    for img, _, _, _ in b["parts"].values():
        count[img] = count.get(img, 0) + 1
    for img, k in cfg.parts:
        assert count.get(img, 0) >= k, (img, count.get(img, 0), k)
    # every net has a class, and the class names are the configuration's
    names = {c[0] for c in cfg.classes}
    assert set(b["classes"]) >= set(signal) and set(b["classes"].values()) <= names


@pytest.mark.parametrize("name", ["c1", "c2", "c4", "c5"])
def test_pads_lie_inside_the_board_and_parts_do_not_overlap(name):
    b = _parse(dsngen.generate(name, 3))
    x0, y0, x1, y1 = b["box"]
    boxes = []
    for ref, (img, px, py, rot) in b["parts"].items():
        pads = []
        for dx, dy in b["images"][img].values():
            if rot in (90, 270):
                dx, dy = -dy, dx
            pads.append((px + dx, py + dy))
            assert x0 < px + dx < x1 and y0 < py + dy < y1, (ref, px + dx, py + dy)
        boxes.append((min(p[0] for p in pads), min(p[1] for p in pads), max(p[0] for p in pads),
                      max(p[1] for p in pads)))
    boxes.sort()
    # pad extents of two parts never intersect (sweep over x)
    for i, a in enumerate(boxes):
        for bb in boxes[i + 1:]:
            if bb[0] > a[2]:
                break
            assert bb[1] > a[3] or a[1] > bb[3], (a, bb)


def test_boards_are_deterministic_per_seed():
    for name in ("c1", "c2"):
        assert dsngen.generate(name, 5) == dsngen.generate(name, 5)
        assert dsngen.generate(name, 5) != dsngen.generate(name, 6)
