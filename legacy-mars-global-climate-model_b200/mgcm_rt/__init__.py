"""Host side of the B200 column radiative transfer for the Legacy Mars GCM.

``mgcm_rt.abi``   ctypes binding of the C ABI in include/mgcm_rt.h
``mgcm_rt.synth`` seeded synthetic column batches (reference input recipe)
``mgcm_rt.data``  data-file locations and formats
"""
from . import data, synth  # noqa: F401

INPUT_LEV = ("plev", "tlev", "pmid", "tmid", "qh2o")
INPUT_LEV1 = ("tauref", "qextrefdst")
INPUT_CLD_LEV1 = ("taurefcld", "qextrefcld")
INPUT_VBAND = ("qxvdst", "qsvdst", "gvdst")
INPUT_IBAND = ("qxidst", "qsidst", "gidst")
INPUT_CLD_VBAND = ("qxvcld", "qsvcld", "gvcld")
INPUT_CLD_IBAND = ("qxicld", "qsicld", "gicld")
INPUT_COL = ("acosz", "als", "albi", "pcol")
OUTPUT_LAY = ("fmnetv", "fluxupv", "fluxdnv", "fmneti", "fluxupi", "fluxdni",
              "suntot", "irtotal", "qrad")
OUTPUT_COL = ("nfluxtopv", "nfluxtopi", "diffvt", "dnvflux", "dndiffv", "dnirflux",
              "fluxsurf")
INOUT_STATE = ("detau", "cumtauv")
