"""Command line compatible with the reference's ``./bench`` (cuda/main.cpp:9-147).

    python -m threadcoarsenedstencilgenerator_b200.cli <neighbourhood> <2D|3D> <range> <coefficients>
        <orientation> <alignment> <CLsize> <maxTime> <cx> <cy> [<cz>] <nx> <ny> [<nz>] [<bx> <by> [<bz>]]

13 / 15 arguments (argv incl. program name) run the exhaustive block sweep in 2D / 3D, 15 / 18
run a single block shape ("profile" mode), exactly as main.cpp dispatches.  The report is the
reference's TSV.  ``--precision f32`` selects single-precision grids (an addition).
"""

from __future__ import annotations

import sys

USAGE = """Unknown arguments, the relevant arguments have to match the generated kernel code.
Usage:
\t\tstencil neighbourhood ('Box' or 'Star')
\t\tdimension ('2D' or '3D')
\t\tstencil range > 0
\t\tcoefficients type ('Jacobi' or 'Variable')
\t\torientation\t('Column' or 'Row')
\t\talignment\t('None', 'Write' or 'Read')
\t\tsize of cache line in units of grid elements
\t\tmaximal runtime for single threadblock size in seconds
\t\tcoarsening factors (x y z[only for 3D])

\t\tgrid size (x y z[only for 3D])

optional for run of single threadblock size:
\t\tthread block size (x y z[only for 3D])
"""


def main(argv=None) -> int:
    argv = list(sys.argv if argv is None else argv)
    precision = "f64"
    if "--precision" in argv:
        i = argv.index("--precision")
        precision = argv[i + 1]
        del argv[i:i + 2]
    argc = len(argv)
    bench2d, profile2d = 13, 15
    bench3d, profile3d = 15, 18
    if not (bench2d <= argc <= profile3d):
        sys.stderr.write(USAGE)
        return 1
    neighbourhood, sdim = argv[1], argv[2]
    try:
        rng, coeff, orient, align = int(argv[3]), argv[4], argv[5], argv[6]
        cl, max_time = int(argv[7]), float(argv[8])
        if sdim == "2D":
            dim = 2
        elif sdim == "3D":
            dim = 3
        else:
            sys.stderr.write("Unknown dimension: %s\n" % sdim + USAGE)
            return 1
        cx, cy = int(argv[9]), int(argv[10])
        cz = 1
        block = None
        if dim == 2 and argc == bench2d:
            grid = (int(argv[11]), int(argv[12]), 1)
        elif dim == 3 and argc == bench3d:
            cz = int(argv[11])
            grid = (int(argv[12]), int(argv[13]), int(argv[14]))
        elif dim == 2 and argc == profile2d:
            grid = (int(argv[11]), int(argv[12]), 1)
            block = (int(argv[13]), int(argv[14]), 1)
        elif dim == 3 and argc == profile3d:
            cz = int(argv[11])
            grid = (int(argv[12]), int(argv[13]), int(argv[14]))
            block = (int(argv[15]), int(argv[16]), int(argv[17]))
        else:
            sys.stderr.write("Dimension and amount of arguments mismatch!\n" + USAGE)
            return 1
    except ValueError as e:
        sys.stderr.write("%s\n%s" % (e, USAGE))
        return 1

    from . import _lib
    from .benchmark import StencilBenchmark

    try:
        b = StencilBenchmark(neighbourhood, dim, align, cl, coeff, orient, rng, (cx, cy, cz), grid, max_time,
                             precision=precision)
        b.init_gpu()
        b.init_benchmark()
        if block is None:
            b.run()
        else:
            b.single_run(*block)
    except (ValueError, MemoryError, _lib.TcsError) as e:
        sys.stderr.write("%s\nExiting!\n" % e)
        return 1
    b.print_results()
    return 0


if __name__ == "__main__":
    sys.exit(main())
