"""Limiter ids understood by the 2D step (src/pyclaw/limiters/tvd.py:74-77 and
the computed GOTO of philim.f90:18-55).  Ids 1-5 select minmod, superbee,
van Leer, MC and Beam-Warming; other positive ids fall through to minmod, as
in the reference's 2D Fortran kernel; 0 leaves a wave family unlimited."""
minmod = 1
superbee = 2
vanleer = 3
MC = 4
beam_warming = 5
