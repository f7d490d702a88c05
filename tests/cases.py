"""Seeded parity cases at sizes the oracle finishes in seconds.

Each case is (mode, Job, frequency list).  The shapes follow the
configurations of the reference runs (source depth, receiver spread,
epicentral grid) scaled down in grid density and frequency count.
"""
import dsmsgt
from dsmsgt import synth


def sh_small(seed=0, imax=32, thdelta=15.0, rdelta=350.0):
    """SH mantle model, 100 km deep source, receivers through the mantle."""
    return dsmsgt.Job(
        synth.param_file(tlen=1638.4, rmin=3500.0, rmax=6300.0, rdelta=rdelta, r0=6271.0,
                         thmin=0.0, thmax=180.0, thdelta=thdelta, imin=0, imax=imax),
        synth.dsm_config(), synth.sh_mantle_model(seed))


def psv_small(seed=0, imax=64, thdelta=15.0, rdelta=500.0, r0=6071.0, rmin=1000.0):
    """PSV Earth model with inner core, fluid outer core and mantle; receivers
    from the inner core to the surface (fluid receivers included)."""
    return dsmsgt.Job(
        synth.param_file(tlen=1638.4, rmin=rmin, rmax=6300.0, rdelta=rdelta, r0=r0,
                         thmin=0.0, thmax=180.0, thdelta=thdelta, imin=0, imax=imax),
        synth.dsm_config(), synth.psv_earth_model(seed))
