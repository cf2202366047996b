"""Reference build configurations — TEST INFRASTRUCTURE ONLY (oracle).

Each entry lists the compile-time macro values written into the reference's
``src/definitions.h`` (reference ``DNS-solver-with-grid-embedding/src/
definitions.h:34-119``) for one oracle build, with ``XDIM = YDIM = 1`` (one
rank, so the decomposition reduces to a periodic single domain).

Names:
  t_*  tiny grids (seconds of CPU) used by the parity tests;
  c1   the plain FP64 channel, coarse 64 x 32 x 64 in (stream, wall-normal,
       span) = reference (xdv, ydv, zdv) = (64, 64, 27) with zds = 8, GR = 2
       (fine block 128 x 8 x 128 per wall, H = 63 fine cells);
  c2   the production channel 256 x 96 x 128 -> (256, 128, 83), zds = 16;
  c3r / c3p  the superhydrophobic channel 384 x 128 x 192 -> (384, 192, 115),
       zds = 16, with streamwise ridges (pitch 48, gas fraction 0.5) or square
       posts (pitch 32, gas fraction 0.75).

``tke``: also build the reference's turbulence-statistics / kinetic-energy
budget program (TKE-budget/computations) for that grid.

Reynolds numbers: for c1 the bulk Reynolds number is chosen so that the fine
relaxation time is 0.52 (Reb = 150 ub H, H = NZs - 2 fine cells); c2/c3 use
Dean's correlation Re_tau = 0.0955 Re_b^(7/8) (Re_b on the full height) for
Re_tau = 180 and 395.
"""

UB = 0.0866034  # reference default bulk velocity (definitions.h:35)


def _h(zdv, zds, gr):
    zdf = zds + 1
    return 2 * zdf + gr * (zdv - 4) + gr - 1 - 2


def _tiny(**kw):
    cfg = dict(Rebs=200.0, ub=UB, zdv=7, ydv=8, xdv=8, TSTR=100, TEND=101, CFL=2.0, gratio=2, zds=4,
               gyplussize=4, wyplussize=4, gxplussize=4, wxplussize=4, XDIM=1, YDIM=1, ITER=50)
    cfg.update(kw)
    return cfg


REF_CONFIGS = {
    # the two configurations with the unmodified main also carry a small uniform
    # grid for its mode -i start
    "t_noslip": _tiny(main=True, xdu=12, ydu=12, zdu=11),
    "t_ridges": _tiny(pattern="RSLIP", main=True, xdu=12, ydu=12, zdu=11),
    "t_posts": _tiny(pattern="PSLIP"),
    "t_span": _tiny(pattern="SSLIP"),
    "t_gr4": _tiny(xdv=8, ydv=4, zdv=7, zds=8, gratio=4, pattern="PSLIP", gxplussize=8, wxplussize=8, tke=True),
    # the filtered fine-to-coarse transfer (FLTR), defined by the reference for
    # GR = 4 (its stencil array holds GR + 1 = 5 planes)
    "t_gr4f": _tiny(xdv=8, ydv=4, zdv=7, zds=8, gratio=4, pattern="PSLIP", gxplussize=8, wxplussize=8, fltr=True,
                    main=True),
    "t_odd": _tiny(xdv=12, ydv=6, zdv=9, zds=6, pattern="RSLIP", gyplussize=6, wyplussize=6, tke=True),
    "c1": dict(Rebs=repr(150.0 * UB * _h(27, 8, 2)), ub=UB, zdv=27, ydv=64, xdv=64, TSTR=0, TEND=1,
               CFL=0.1, gratio=2, zds=8, gyplussize=4, wyplussize=4, gxplussize=4, wxplussize=4,
               XDIM=1, YDIM=1, tke=True),
    "c2": dict(Rebs=5533.0, ub=UB, zdv=83, ydv=128, xdv=256, TSTR=0, TEND=1, CFL=0.1, gratio=2,
               zds=16, gyplussize=4, wyplussize=4, gxplussize=4, wxplussize=4, XDIM=1, YDIM=1, tke=True),
    "c3r": dict(Rebs=13585.0, ub=UB, zdv=115, ydv=192, xdv=384, TSTR=0, TEND=1, CFL=0.1, gratio=2,
                zds=16, gyplussize=24, wyplussize=24, gxplussize=16, wxplussize=16, XDIM=1, YDIM=1,
                pattern="RSLIP"),
    "c3p": dict(Rebs=13585.0, ub=UB, zdv=115, ydv=192, xdv=384, TSTR=0, TEND=1, CFL=0.1, gratio=2,
                zds=16, gyplussize=16, wyplussize=16, gxplussize=16, wxplussize=16, XDIM=1, YDIM=1,
                pattern="PSLIP"),
}
