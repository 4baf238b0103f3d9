"""The per-GPU launch-parameter file (CPU only): the file name the tuner
writes is the one the library reads (csrc/tuning.cu, file_stem), and the
shipped B200 file holds only parameters and values the tuner searches."""
import os
import re

from pacman_b200 import tune


def _read(path):
    out = {}
    for line in open(path):
        line = line.split("#", 1)[0]
        if "=" in line:
            k, v = (x.strip() for x in line.split("=", 1))
            out[k] = v
    return out


def test_file_name_matches_the_library():
    p = tune.conf_path("NVIDIA B200")
    assert p.endswith(os.path.join("pacman_b200", "tuning", "NVIDIA_B200.conf"))
    # The library keeps [A-Za-z0-9.-] and maps everything else to '_'.
    assert os.path.basename(tune.conf_path("NVIDIA GB200 (x)")) == "NVIDIA_GB200__x_.conf"


def test_shipped_b200_file_is_in_the_search_space():
    conf = _read(tune.conf_path("NVIDIA B200"))
    assert set(conf) == set(tune.SPACE)
    for k, v in conf.items():
        assert v in tune.SPACE[k], (k, v)


def test_library_parses_every_tuned_key():
    src = open(os.path.join(os.path.dirname(tune.__file__), "csrc", "tuning.cu")).read()
    parsed = set(re.findall(r'key == "(PACMAN_B200_\w+)"', src))
    assert set(tune.SPACE) <= parsed
