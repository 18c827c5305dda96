"""The C-ABI library without a GPU: it loads, exports every function include/mclics_b200.h declares, fails
cleanly (status code + message, no crash, no exit) where a device is needed, and runs the reference's input
validation (src/io.cpp:381-475, tests/run_checks.py:326-380) before touching the device or any file."""
import os
import re

import pytest

from helpers import M, base, input_text, plus

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HAS_GPU = False
try:
    import torch

    HAS_GPU = torch.cuda.is_available()
except Exception:
    pass


def declared_functions():
    text = open(os.path.join(ROOT, "include", "mclics_b200.h")).read()
    return sorted(set(re.findall(r"\b(mcl_[a-z_]+)\s*\(", text)))


def test_library_exports_every_declared_function():
    L = M.lib()
    names = declared_functions()
    assert len(names) >= 20
    for n in names:
        assert hasattr(L, n), n
    assert M.version().startswith("mclics_b200")


def test_struct_layouts_match_header(tmp_path):
    """ctypes mirrors of the C structs have the sizes and field offsets a C compiler gives the header."""
    import ctypes
    import subprocess
    src = tmp_path / "sz.c"
    checks = []
    for cname, py in (("mcl_model", M.CModel), ("mcl_replica", M.CReplica), ("mcl_observables", M.CObservables),
                      ("mcl_tuning", M.CTuning), ("mcl_extras", M.CExtras)):
        checks.append('printf("%%s %%zu\\n", "%s", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            checks.append('printf("%%s.%%s %%zu\\n", "%s", "%s", offsetof(%s, %s));' % (cname, f, cname, f))
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "mclics_b200.h"\nint main(void){%s return 0;}\n'
                   % "\n".join(checks))
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.split("\n") if l)
    for cname, py in (("mcl_model", M.CModel), ("mcl_replica", M.CReplica), ("mcl_observables", M.CObservables),
                      ("mcl_tuning", M.CTuning), ("mcl_extras", M.CExtras)):
        assert int(out[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(out["%s.%s" % (cname, f)]) == getattr(py, f).offset, (cname, f)


@pytest.mark.skipif(HAS_GPU, reason="checks the no-device path")
def test_create_without_device_reports_error():
    with pytest.raises(M.McLicsError) as ei:
        M.Engine(M.Model(), [M.Replica(8, 8, 8)])
    assert ei.value.code in (8, 2)


def test_create_rejects_bad_arguments_before_device():
    with pytest.raises(M.McLicsError) as ei:
        M.Engine(M.Model(), [M.Replica(5, 8, 8)])  # odd periodic size
    assert ei.value.code == 1 and "even number of sites" in str(ei.value)
    with pytest.raises(M.McLicsError):
        M.Engine(M.Model(), [M.Replica(8, 8, 8, geometry="slab")])  # slab without anchoring


@pytest.mark.parametrize("sizes,text", [
    ((0, 8, 8), "grid sizes must be >= 1"),
    ((8, 8, 0), "grid sizes must be >= 1"),
    ((-2, 8, 8), "grid sizes must be >= 1"),
    ((4096, 4096, 4096), "more than 2^32 sites"),   # the Philox site counter is 32 bits wide
    ((65536, 65536, 2), "more than 2^32 sites"),
], ids=["empty_x", "empty_z", "negative", "cube_4096", "flat_65536"])
def test_create_rejects_empty_and_oversized_lattices(sizes, text):
    with pytest.raises(M.McLicsError) as ei:
        M.Engine(M.Model(), [M.Replica(*sizes)])
    assert ei.value.code == 1 and text in str(ei.value)


def test_create_rejects_an_empty_batch():
    with pytest.raises(M.McLicsError) as ei:
        M.Engine(M.Model(), [])
    assert ei.value.code == 1 and "no replicas" in str(ei.value)


ERRORS = [
    ("odd_periodic", base(Nx=5), "requires an even number of sites"),
    ("wrong_dT", base(Ti=0.5, Tf=1.0, dT=-0.1), "does not lead from Ti"),
    ("unknown_parameter", plus(base(), "Tff 0.1"), "Unknown parameter"),
    ("unknown_anchoring", plus(base(Nz=6, geometry="slab"), "anchoring_type 0 strong", "W 0 1",
                               "anchoring_type 1 rp", "W 1 1", "theta_s 1 90", "phi_s 1 0"), "not implemented"),
    ("missing_anchoring", plus(base(Nz=6, geometry="slab"), "anchoring_type 0 homeotropic", "W 0 1"),
     "anchoring_type 1 is not defined"),
    ("ghrl_constants", base(potential="ghrl", k11=5, k22=1, k33=1), "needs k11 < 3 k22 + k33"),
    ("negative_temperature", base(Ti=-0.1, Tf=-0.1), "Ti must be >= 0"),
    ("bad_value", plus(base(), "MCS many"), "Invalid value for parameter"),
    ("unknown_mode", base(evol="wobbleGPU"), "not implemented"),
    ("zero_field_dir", base(elecA=0.5), "field direction"),
]


@pytest.mark.parametrize("name,params,text", ERRORS, ids=[e[0] for e in ERRORS])
def test_input_errors_leave_old_output(name, params, text, tmp_path, capfd):
    d = str(tmp_path)
    with open(os.path.join(d, "input.txt"), "w") as f:
        f.write(input_text(params))
    with open(os.path.join(d, "po.dat"), "w") as f:
        f.write("old results\n")
    cwd = os.getcwd()
    os.chdir(d)
    try:
        with pytest.raises(M.McLicsError) as ei:
            M.run_input_file("input.txt")
    finally:
        os.chdir(cwd)
    err = capfd.readouterr().err
    assert text in err, err
    assert ei.value.code in (1, 5)
    assert open(os.path.join(d, "po.dat")).read() == "old results\n"


def test_mlp_struct_is_the_flat_parameter_vector(tmp_path):
    import subprocess
    src = tmp_path / "m.c"
    src.write_text('#include <stdio.h>\n#include "mclics_b200.h"\nint main(void){printf("%zu\\n", sizeof(mcl_mlp));'
                   'return 0;}\n')
    exe = tmp_path / "m"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    assert int(out) == 4 * M.N_MLP_PARAMS
