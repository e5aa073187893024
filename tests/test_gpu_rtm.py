"""Media modes and reverse-time migration (qvti_set_media, qvti_set_injection,
qvti_rtm_shot) -- the options the reference's host program declares and
does not implement (viscoelas_3D.cpp:1-3, 42-65, 223-229).

* media: a pulse travelling 20 cells through Qp = 30 arrives weakest in the
  viscoelastic medium, stronger with the loss terms off (dispersion only),
  strongest with them reversed (Q-compensated); the lossless medium matches
  dispersion-only in amplitude.
* RTM: the reflections of a two-layer model (records of the model minus
  those of its top layer alone) migrated with the top layer's velocity image
  the interface at its depth.
* Q-compensated RTM: with attenuating data, compensating both propagations
  brings the reflector's image amplitude back toward that of lossless data
  migrated losslessly; where the compensation blows up the shot says so.
"""
import numpy as np
import pytest

import qvti_cases as qc

pytestmark = pytest.mark.gpu


def _pulse_case(nt=160):
    n = (64, 64, 64)
    c = qc.homogeneous_case(n=n, pml=10, d=(10.0, 10.0, 10.0), dt=1e-3, nt=nt, f0=25.0, qp=30.0, qs=15.0,
                            src=(32, 32, 24), r_iz=44)
    return c


def test_media_change_the_amplitude_as_they_should(qvti):
    c = _pulse_case()
    amp = {}
    for name, media in (("visco", qvti.MEDIA_VISCOELASTIC), ("disp", qvti.MEDIA_DISPERSION_ONLY),
                        ("lossless", qvti.MEDIA_LOSSLESS), ("comp", qvti.MEDIA_Q_COMPENSATED)):
        r = qvti.run_case(c, src_type=qvti.SRC_EXPLOSIVE, media=media)["rec"]
        assert np.isfinite(r).all()
        amp[name] = float(np.abs(r[2][:, 32]).max())  # vz straight below the source
    assert amp["visco"] < amp["disp"] < amp["comp"], amp
    assert 0.8 < amp["lossless"] / amp["disp"] < 1.25, amp
    # the same attenuation removed and added back, to first order
    g_loss, g_comp = amp["disp"] / amp["visco"], amp["comp"] / amp["disp"]
    assert 0.6 < g_comp / g_loss < 1.6, amp


def _layered(n=(64, 64, 96), z_if=50, qp=1000.0, two=True):
    c = qc.homogeneous_case(n=n, pml=10, d=(10.0, 10.0, 10.0), dt=1e-3, nt=420, f0=25.0, vp=2500.0, vs=1445.0,
                            rho=2000.0, qp=qp, qs=qp / 2, src=(32, 32, 14), r_iz=12)
    if two:
        for k, v in (("velp", 3500.0), ("vels", 2020.0), ("rho", 2300.0)):
            c[k] = c[k].copy()
            c[k][:, :, z_if:] = v
    gx = np.arange(0, n[0], 2, dtype=np.int32)
    c["r_ix"] = np.repeat(gx, gx.size)
    c["r_iy"] = np.tile(gx, gx.size)
    c["rnx_max"], c["rny_max"] = gx.size, gx.size
    return c


def _reflections(qvti, media, qp):
    """Records of the two-layer model minus those of its top layer alone."""
    full = qvti.run_case(_layered(qp=qp), src_type=qvti.SRC_EXPLOSIVE, media=media)["rec"]
    top = qvti.run_case(_layered(qp=qp, two=False), src_type=qvti.SRC_EXPLOSIVE, media=media)["rec"]
    return full - top


def _depth_profile(image, pml=10):
    """Mean |image| over the central 16 x 16 columns, per depth index."""
    return np.abs(image[24:40, 24:40, :]).mean(axis=(0, 1))


def test_rtm_images_the_interface(qvti):
    z_if = 50
    obs = _reflections(qvti, qvti.MEDIA_VISCOELASTIC, 1000.0)
    assert np.abs(obs).max() > 0
    mig = _layered(qp=1000.0, two=False)  # migration model: the top layer's velocity
    xc, nrm = qvti.rtm_shot(mig, obs, media=qvti.MEDIA_VISCOELASTIC, snap_every=5, src_type=qvti.SRC_EXPLOSIVE)
    assert np.isfinite(xc).all() and np.isfinite(nrm).all()
    for im in (xc, nrm):
        prof = _depth_profile(im)
        zs = np.arange(24, 96 - 10)  # below the source and receivers, above the bottom C-PML
        z_peak = int(zs[np.argmax(prof[zs])])
        assert abs(z_peak - z_if) <= 3, (z_peak, prof[zs].round(8))


def test_q_compensated_rtm_restores_the_reflector_amplitude(qvti):
    # Qp 100, Qs 50: the reflection loses about a fifth of its amplitude each
    # way at 25 Hz, and compensation by sign reversal stays well posed over
    # the 420 steps (at Qp 30 it blows up: test below)
    z_if, q = 50, 100.0
    lossless = _reflections(qvti, qvti.MEDIA_LOSSLESS, q)
    visco = _reflections(qvti, qvti.MEDIA_VISCOELASTIC, q)
    mig = _layered(qp=q, two=False)
    amp = {}
    for name, obs, media in (("ref", lossless, qvti.MEDIA_LOSSLESS), ("visco", visco, qvti.MEDIA_VISCOELASTIC),
                             ("comp", visco, qvti.MEDIA_Q_COMPENSATED)):
        xc, _ = qvti.rtm_shot(mig, obs, media=media, snap_every=5, src_type=qvti.SRC_EXPLOSIVE)
        assert np.isfinite(xc).all()
        amp[name] = float(_depth_profile(xc)[z_if - 3:z_if + 4].max())
    assert amp["visco"] < amp["comp"], amp
    assert abs(amp["comp"] - amp["ref"]) < abs(amp["visco"] - amp["ref"]), amp


def test_q_compensation_that_blows_up_is_reported(qvti):
    """Sign-reversed loss terms amplify the high wavenumbers too; through Qp 30
    over 420 steps the compensated propagation turns non-finite, and the
    shot reports QVTI_ERR_NONFINITE instead of returning an image of NaN."""
    visco = _reflections(qvti, qvti.MEDIA_VISCOELASTIC, 30.0)
    with pytest.raises(qvti.QvtiError, match="non-finite"):
        qvti.rtm_shot(_layered(qp=30.0, two=False), visco, media=qvti.MEDIA_Q_COMPENSATED, snap_every=5,
                      src_type=qvti.SRC_EXPLOSIVE)
