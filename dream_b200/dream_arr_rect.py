"""Module named as the reference's ``dream_arr_rect`` extension
(python/src/py_dream_arr_rect.cc): ``from dream_b200 import dream_arr_rect as
dar; dar.dream_arr_rect(...)``. The implementation is in dreamrect.py."""
from .dreamrect import APOD_METHODS, FOC_METHODS, STEER_METHODS, dream_arr_rect  # noqa: F401
