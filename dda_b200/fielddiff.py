"""Compare two result files by their normalised RMS difference, the check the
reference's test scripts run on its outputs (DDA/FieldDiff.cpp).

    python -m dda_b200.fielddiff [--print-only | --max-error 1e-4] FILE1 FILE2 [LEN[:FACTOR1] ...]

Text files (the reference's layout: one header line, then whitespace-separated
numbers; DDA/FieldDiff.cpp:65-130): the columns of each line fall into groups of
LEN values, the values of FILE1 in a group scaled by FACTOR1 (default 1).  For
each group, with d1 from FILE1 and d2 from FILE2 over all lines,

    normalised = sqrt(sum (d2 - d1)^2 / ((sum d1^2 + sum d2^2) / 2))

(DDA/FieldDiff.cpp:189-192).  Files of different lengths, or lines with extra
fields, are an error (exit 1); so is a group whose normalised difference is not
below --max-error (default 1e-4), unless --print-only, which prints the
normalised values alone.

MATLAB-style HDF5 files (the .hdf5 outputs, read by `matfile`): without groups,
one group over the real and imaginary parts of the file's data: Field.Data of
field files, JonesFarField.Data or MuellerFarField.Data of far-field files, the
CrossSection values of cross-section files.  This is the same metric on the
values the text files hold, without their rounding to 10 digits.
"""
import math
import sys

import numpy as np

from . import matfile


def normalised_rms(a, b, factor1=1.0):
    """sqrt(sum (b - f a)^2 / ((sum (f a)^2 + sum b^2) / 2)) over the real
    and imaginary parts of a (scaled by f) and b."""
    a = np.asarray(a) * factor1
    b = np.asarray(b)
    x = np.concatenate([np.real(a).ravel(), np.imag(a).ravel()])
    y = np.concatenate([np.real(b).ravel(), np.imag(b).ravel()])
    den = (np.dot(x, x) + np.dot(y, y)) / 2
    return math.sqrt(np.dot(y - x, y - x) / den) if den > 0 else float("nan")


def _lines(path):
    with open(path) as f:
        f.readline()  # the header line is skipped
        return [l.split() for l in f if l.strip()]


def compare_text(path1, path2, groups):
    """Per group (len, factor1): (values, squared difference, squared sum 1,
    squared sum 2, normalised); and the number of lines compared."""
    l1, l2 = _lines(path1), _lines(path2)
    if len(l1) != len(l2):
        longer, shorter = (path1, path2) if len(l1) > len(l2) else (path2, path1)
        raise ValueError("`%s' is longer than `%s'" % (longer, shorter))
    width = sum(n for n, _ in groups)
    for i, (a, b) in enumerate(zip(l1, l2)):
        for path, row in ((path1, a), (path2, b)):
            if len(row) > width:
                raise ValueError("`%s' has extra fields on line %d" % (path, i + 2))
            if len(row) < width:
                raise ValueError("`%s' has too few fields on line %d" % (path, i + 2))
    d1 = np.array(l1, dtype=np.float64).reshape(len(l1), width)
    d2 = np.array(l2, dtype=np.float64).reshape(len(l2), width)
    out, c = [], 0
    for n, factor in groups:
        x, y = d1[:, c:c + n] * factor, d2[:, c:c + n]
        c += n
        diff, s1, s2 = float(np.sum((y - x) ** 2)), float(np.sum(x * x)), float(np.sum(y * y))
        norm = math.sqrt(diff / ((s1 + s2) / 2)) if s1 + s2 > 0 else float("nan")
        out.append((x.size, diff, s1, s2, norm))
    return out, len(l1)


def hdf5_values(path):
    """The data a result file holds, as one array."""
    f = matfile.load(path)
    kind = f.get("Type")
    if kind == "DDAField":
        return np.asarray(f["Field"]["Data"])
    if kind == "JonesFarField":
        return np.asarray(f["JonesFarField"]["Data"])
    if kind == "MuellerFarField":
        return np.asarray(f["MuellerFarField"]["Data"])
    if kind == "CrossSection":
        cs = f["CrossSection"]
        return np.array([cs[k][0] for k in ("Cext", "Cabs", "Csca", "Qext", "Qabs", "Qsca")])
    raise ValueError("`%s': no comparable data (Type %r)" % (path, kind))


def main(argv=None):
    args = list(sys.argv[1:] if argv is None else argv)
    print_only, max_error = False, 1e-4
    if args[:1] == ["--print-only"]:
        print_only, args = True, args[1:]
    elif args[:1] == ["--max-error"] and len(args) >= 2:
        max_error, args = float(args[1]), args[2:]
    if len(args) < 2:
        sys.stderr.write("Usage: python -m dda_b200.fielddiff [--print-only | --max-error 1e-4] <filename1> "
                         "<filename2> <group1len>:<group1factor1> ...\n")
        return 1
    f1, f2 = args[0], args[1]
    try:
        if matfile.is_hdf5(f1) and matfile.is_hdf5(f2) and len(args) == 2:
            a, b = hdf5_values(f1), hdf5_values(f2)
            if a.shape != b.shape:
                raise ValueError("`%s' holds %s values, `%s' %s" % (f1, a.shape, f2, b.shape))
            norms = [normalised_rms(a, b)]
            report = ["Read %d values, normalized error is %.15f%%" % (2 * a.size, norms[0] * 100)]
        else:
            groups = []
            for g in args[2:]:
                parts = g.split(":")
                if len(parts) not in (1, 2):
                    raise ValueError("bad group `%s'" % g)
                groups.append((int(parts[0]), float(parts[1]) if len(parts) > 1 else 1.0))
            if not groups:
                raise ValueError("text files need column groups")
            res, n = compare_text(f1, f2, groups)
            norms = [r[4] for r in res]
            report = ["Read %d values for group %d on %d lines, got a squared difference of %.10g, avg %.10g, "
                      "squared sum 1 is %.10g, squared sum 2 is %.10g, normalized error is %.15f%%"
                      % (r[0], i, n, r[1], r[1] / max(r[0], 1), r[2], r[3], r[4] * 100) for i, r in enumerate(res)]
    except (OSError, ValueError, KeyError, matfile.MatFileError) as e:
        sys.stderr.write("%s\n" % e)
        return 1
    if print_only:
        for v in norms:
            print("%.15f" % v)
        return 0
    for line in report:
        print(line)
    for i, v in enumerate(norms):
        if not v < max_error:
            sys.stderr.write("Avg difference of group %d too large\n" % i)
            return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
