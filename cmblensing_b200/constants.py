"""Constants and enums of cmb_lensing/constants.py:5-39, restated for the B200 engine."""
import math

ARCMIN_PER_DEGREE = 60
INVERSE_LENSE = -1
FORWARD_LENSE = +1
NSIDE_DEFAULT = 256
THETA_PIX_DEFAULT = 2.5
PIX_WIDTH_DEFAULT = math.radians(THETA_PIX_DEFAULT / ARCMIN_PER_DEGREE)
SUPPORTED_NSIDE = (64, 128, 256, 512, 1024)


class Parametrization:
    T = 0
    QU = 1
    EB = 2


class Basis:
    MAP = 0
    FOURIER = 1


class Polarity:
    I = "I"
    P = "P"
    IP = "IP"
