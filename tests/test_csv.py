"""CPU tests of the ThunderStorm CSV writer (data/PLocalization.java:224-306)."""
import numpy as np


def test_java_double_format(zpkg):
    jd = zpkg.java_double
    assert jd(0.0) == "0.0"
    assert jd(1.0) == "1.0"
    assert jd(-1.235) == "-1.235"
    assert jd(123.456) == "123.456"
    assert jd(1234567.0) == "1234567.0"
    assert jd(12345678.0) == "1.2345678E7"
    assert jd(0.001) == "0.001"
    assert jd(0.0001) == "1.0E-4"
    assert jd(2500.5) == "2500.5"


def test_csv_header_rows_and_flooring(zpkg, tmp_path):
    dt = np.dtype([(c, np.int32 if c in ("id", "frame", "candidate", "fit_status") else np.float64)
                   for c in zpkg.LOC_COLUMNS])
    locs = np.zeros(2, dtype=dt)
    # the last two fields (candidate index, fit status) are not CSV columns
    locs[0] = (0, 3, 1234.56789, -0.0004, 250.0, 2999.9999, 20.5, 1.02345, 5.5555, 6.0, 12.34567, 17, 1)
    locs[1] = (1, 4, 0.0, 0.0, -100.0, 100.0, 1.0, 0.5, 1.0, 1.0, 1.0, 2, 2)
    path = str(tmp_path / "loc.csv")
    zpkg.write_csv(path, locs)
    lines = open(path).read().splitlines()
    assert lines[0] == ("id,frame,x [nm],y [nm],z [nm],intensity,background,chi2,crlbX,crlbY,crlbZ,driftX,driftY,"
                        "driftZ,occurrenceMerging")
    # values floored to 1e-3 (PLocalization.java:59-72)
    assert lines[1] == "0,3,1234.567,-0.001,250.0,2999.999,20.5,1.023,5.555,6.0,12.345,0.0,0.0,0.0,1"
    assert lines[2] == "1,4,0.0,0.0,-100.0,100.0,1.0,0.5,1.0,1.0,1.0,0.0,0.0,0.0,1"
    zpkg.write_csv(path, locs[:1], append=True)
    assert len(open(path).read().splitlines()) == 4
