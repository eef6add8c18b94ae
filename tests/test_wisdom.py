"""Autotuning records ("wisdom") file handling, without a GPU: import of a
well-formed file and export give back the same records; malformed files
are refused and change nothing; forget drops every record."""
import pytest

import mcfft_b200 as mc

HEADER = "mcfft-wisdom 1\n"
RECS = [
    "NVIDIA B200\t148\tL1024 c1 t1 i1024,1,1048576 o1,1024,1048576 n1024,64 h1,1 N1048576\t16384",
    "NVIDIA B200\t148\tL1024 c0 t0 i1,1024,1048576 o1024,1,1048576 n1024,64 h1,1 N0\t8192",
    "Other GPU\t132\tL256 c0 t0 i1,256,65536 o1,256,65536 n1,16 h1,1 N0\t16384",
]


@pytest.fixture(autouse=True)
def clean():
    mc.wisdom_forget()
    yield
    mc.wisdom_forget()


def write(path, text):
    path.write_text(text)
    return str(path)


def records(path):
    lines = path.read_text().splitlines()
    assert lines[0] == HEADER.strip()
    return lines[1:]


def test_import_export_round_trip(tmp_path):
    src = write(tmp_path / "w.txt", HEADER + "".join(r + "\n" for r in RECS))
    mc.wisdom_import(src)
    out = tmp_path / "out.txt"
    mc.wisdom_export(str(out))
    assert records(out) == RECS


def test_import_replaces_same_key_and_accepts_missing_final_newline(tmp_path):
    mc.wisdom_import(write(tmp_path / "a.txt", HEADER + RECS[0] + "\n"))
    changed = RECS[0].rsplit("\t", 1)[0] + "\t8192"
    mc.wisdom_import(write(tmp_path / "b.txt", HEADER + changed))
    out = tmp_path / "out.txt"
    mc.wisdom_export(str(out))
    assert records(out) == [changed]


@pytest.mark.parametrize("text", [
    "mcfft-wisdom 2\n" + RECS[0] + "\n",                       # unknown version
    RECS[0] + "\n",                                            # no header
    HEADER + RECS[0].replace("\t16384", "\t4096") + "\n",      # unsupported tile size
    HEADER + RECS[0].replace("\t16384", "\tx") + "\n",         # not a number
    HEADER + "NVIDIA B200\t148\t16384\n",                      # missing field
    HEADER + RECS[1] + "\n" + "z" * 5000 + "\n",               # overlong line
    "",                                                        # empty file
])
def test_malformed_file_refused_and_changes_nothing(tmp_path, text):
    mc.wisdom_import(write(tmp_path / "good.txt", HEADER + RECS[2] + "\n"))
    with pytest.raises(mc.McfftError) as ei:
        mc.wisdom_import(write(tmp_path / "bad.txt", text))
    assert ei.value.code == mc.INVALID_VALUE
    out = tmp_path / "out.txt"
    mc.wisdom_export(str(out))
    assert records(out) == [RECS[2]]


FS = "NVIDIA B200\t148\tfourstep n%d b1 p0 f0\t%s"


def test_decomposition_records(tmp_path):
    """1D decomposition records: lg n1 of a four-step split (4..13), -1 for
    three passes, -2 for one two-column pass; nothing else."""
    good = [FS % (1 << 20, "10"), FS % (1 << 24, "-1"), FS % (8192, "-2")]
    mc.wisdom_import(write(tmp_path / "w.txt", HEADER + "".join(r + "\n" for r in good)))
    out = tmp_path / "out.txt"
    mc.wisdom_export(str(out))
    assert records(out) == good
    for bad in ("3", "14", "-3", "0", "16384"):
        with pytest.raises(mc.McfftError) as ei:
            mc.wisdom_import(write(tmp_path / "bad.txt", HEADER + FS % (1 << 20, bad) + "\n"))
        assert ei.value.code == mc.INVALID_VALUE
    mc.wisdom_export(str(out))
    assert records(out) == good


def test_missing_file_and_forget(tmp_path):
    with pytest.raises(mc.McfftError):
        mc.wisdom_import(str(tmp_path / "nope.txt"))
    mc.wisdom_import(write(tmp_path / "w.txt", HEADER + RECS[0] + "\n"))
    mc.wisdom_forget()
    out = tmp_path / "out.txt"
    mc.wisdom_export(str(out))
    assert records(out) == []
