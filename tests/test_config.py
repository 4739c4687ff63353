"""spsim.conf parsing and writing through the library's reference-shaped
entry points, against the reference's own read/write (golden fixtures)."""
import json
import os
import subprocess
import sys

import pytest

from conftest import GOLDEN, ROOT
from spsim_b200 import spsim_pybackend as B

CONF = os.path.join(GOLDEN, "config")
OPTION_FIELDS = ["input_type", "pdb_filename", "box_type", "box_dimension", "b_factor", "euler_orientation",
                 "random_orientation", "n_patterns", "vectorize", "delta_atoms", "use_cuda", "wavelength_samples",
                 "random_seed", "output_photons", "output_count", "verbosity_level", "crystal_size", "crystal_cell"]


def _val(v):
    if isinstance(v, bytes):
        return v.decode()
    if hasattr(v, "__len__") and not isinstance(v, str):
        return [float(x) for x in v]
    return v


# The golden files come from the reference compiled without CUDA, whose
# set_defaults gives use_cuda = 0 (src/config.c:54-58); this library is always
# a CUDA build, whose default is 1.  Files that do not set the key differ there.
CUDA_DEFAULT_DIFFERS = {"example", "defaults"}


def _expected_text(name):
    text = open(os.path.join(CONF, name + ".confout")).read()
    if name in CUDA_DEFAULT_DIFFERS:
        assert "use_cuda = 0;" in text
        text = text.replace("use_cuda = 0;", "use_cuda = 1;")
    return text


@pytest.mark.parametrize("name", ["example", "quirks"])
def test_read_then_write_matches_reference_byte_for_byte(tmp_path, name):
    o = B.set_defaults()
    B.read_options_file(os.path.join(CONF, name + ".conf"), o)
    out = tmp_path / (name + ".confout")
    B.write_options_file(str(out), o)
    assert out.read_text() == _expected_text(name)


def test_defaults_write_matches_reference(tmp_path):
    o = B.set_defaults()
    out = tmp_path / "d.confout"
    B.write_options_file(str(out), o)
    assert out.read_text() == _expected_text("defaults")


@pytest.mark.parametrize("name", ["example", "quirks", "defaults"])
def test_parsed_values_match_reference(name):
    ref = json.load(open(os.path.join(CONF, "parsed.json")))[name]
    if name in CUDA_DEFAULT_DIFFERS:
        ref["use_cuda"] = 1
    o = B.set_defaults()
    if name != "defaults":
        B.read_options_file(os.path.join(CONF, name + ".conf"), o)
    oc = o.contents
    for k in OPTION_FIELDS:
        v = _val(getattr(oc, k))
        assert v == pytest.approx(ref[k]) if not isinstance(v, str) else v == ref[k], k
    for k, v in ref.items():
        if k.startswith("detector."):
            assert _val(getattr(oc.detector.contents, k.split(".", 1)[1])) == pytest.approx(v), k
        if k.startswith("experiment."):
            assert _val(getattr(oc.experiment.contents, k.split(".", 1)[1])) == pytest.approx(v), k
    cf = oc.chem_formula.contents
    assert [[cf.atomic_number[i], cf.quantity[i]] for i in range(cf.n_elements)] == ref["chem_formula"]


def test_integer_literal_for_float_key_reads_as_zero():
    o = B.set_defaults()
    B.read_options_file(os.path.join(CONF, "quirks.conf"), o)
    assert o.contents.detector.contents.distance == 0.0  # "detector_distance = 1;"


@pytest.mark.parametrize("text", ["a = 5.;", "a = 1e5;", "a = 1\nb = 2;", "a = 1, b = 2;", "_a = 1;", "g = { x = 1; }"])
def test_syntax_errors_exit_like_the_reference(tmp_path, text):
    # the reference's libconfig rejects these forms and read_options_file exits(1) (src/config.c:98-102)
    p = tmp_path / "bad.conf"
    p.write_text(text + "\n")
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from spsim_b200 import spsim_pybackend as B\n"
            "o = B.set_defaults(); B.read_options_file(%r, o); print('parsed')") % (ROOT, str(p))
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert r.returncode == 1 and "Error parsing" in r.stderr, (r.returncode, r.stderr)


@pytest.mark.parametrize("text", ["a : 1.5;", "a = .5;", "a = -1.25e-3;", "a = 0x1F;", "a = (1, 2.0);",
                                  "a = [1, 2];", 'a = "x" "y";', "a = TRUE;", "g = { x = 1; };", "a-b = 1;"])
def test_accepted_forms(tmp_path, text):
    p = tmp_path / "ok.conf"
    p.write_text(text + "\n")
    o = B.set_defaults()
    B.read_options_file(str(p), o)
