"""The generated constant table of 128th roots of unity (minfft_b200/csrc/roots128.h)
used by the axis-pass load and store stages: regenerating it gives the committed
text, and every value is the correctly rounded cos / -sin of 2*pi*m/128."""
import importlib.util
import math
import os
import struct
from decimal import Decimal

import numpy as np

CSRC = os.path.join(os.path.dirname(__file__), "..", "minfft_b200", "csrc")


def load_gen():
    spec = importlib.util.spec_from_file_location("gen_roots128", os.path.join(CSRC, "gen_roots128.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def parse(text, name):
    body = text.split(name + "[kCount] = {")[1].split("};")[0]
    return [float.fromhex(v.strip().rstrip("f")) for v in body.replace("\n", "").split(",")]


def test_header_is_current():
    gen = load_gen()
    with open(os.path.join(CSRC, "roots128.h")) as f:
        assert f.read() == gen.render()


def test_values_correctly_rounded():
    gen = load_gen()
    with open(os.path.join(CSRC, "roots128.h")) as f:
        text = f.read()
    re_d, im_d = parse(text, "kReD"), parse(text, "kImD")
    re_f, im_f = parse(text, "kReF"), parse(text, "kImF")
    assert len(re_d) == len(im_d) == len(re_f) == len(im_f) == 32
    for m in range(32):
        c, s = gen.cos_sin(2 * gen.PI * m / 128)
        a = 2 * math.pi * m / 128
        assert abs(re_d[m] - math.cos(a)) < 1e-15 and abs(im_d[m] + math.sin(a)) < 1e-15
        for got, exact in ((re_d[m], c), (im_d[m], -s)):
            # nearest double: no neighbour is closer to the exact value
            for nb in (np.nextafter(got, -2.0), np.nextafter(got, 2.0)):
                assert abs(Decimal(got) - exact) <= abs(Decimal(float(nb)) - exact)
        for got, exact in ((re_f[m], c), (im_f[m], -s)):
            assert struct.unpack("f", struct.pack("f", got))[0] == got  # a binary32 value
            g32 = np.float32(got)
            for nb in (np.nextafter(g32, np.float32(-2)), np.nextafter(g32, np.float32(2))):
                assert abs(Decimal(got) - exact) <= abs(Decimal(float(nb)) - exact)
    assert re_d[0] == 1.0 and im_d[0] == 0.0 and re_d[16] == -im_d[16]
