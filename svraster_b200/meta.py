"""Constants of the ``svraster_cuda.meta`` module (cuda/svraster_cuda/meta.py:14-31, values
from cuda/src/config.h:14-35)."""

MAX_NUM_LEVELS = 16
STEP_SZ_SCALE = 100.0

VoxGeoModes = dict(
    triinterp=2,
    triinterp1=1,
    triinterp3=3,
)

DensityModes = dict(
    exp_linear_11=0,
    sdf=1,
)

CamModes = dict(
    persp=0,
    ortho=10,
)
