"""Input checks of the alpha path, with the reference's semantics.

``trimap_split`` (pymatting/util/util.py:439-525) and ``sanity_check_image``
(util.py:528-580) are boundary functions: they classify a host trimap into
boolean masks and warn about suspicious inputs. They return host arrays, as
the reference's do; the device side builds its masks with its own kernel
(``_device_trimap_masks``).
"""

import warnings

import numpy as np

__all__ = ["trimap_split", "sanity_check_image"]


def trimap_split(trimap, flatten=True, bg_threshold=0.1, fg_threshold=0.9):
    """Split a trimap into foreground, background, known and unknown masks.

    Foreground: ``trimap >= fg_threshold``; background: ``trimap <=
    bg_threshold``; everything else is unknown. Raises ``ValueError`` when
    either class is empty and warns about values outside [0, 1] or an
    unexpected dtype, like the reference.
    """
    if flatten:
        trimap = trimap.flatten()
    min_value = trimap.min()
    max_value = trimap.max()
    if min_value < 0.0:
        warnings.warn("Trimap values should be in [0, 1], but trimap.min() is %s." % min_value,
                      stacklevel=3)
    if max_value > 1.0:
        # The reference reports min_value in this message as well.
        warnings.warn("Trimap values should be in [0, 1], but trimap.max() is %s." % min_value,
                      stacklevel=3)
    if trimap.dtype not in [np.float32, np.float64]:
        warnings.warn(
            "Unexpected trimap.dtype %s. Are you sure that you do not want to use np.float32 "
            "or np.float64 instead?" % trimap.dtype, stacklevel=3)
    is_fg = trimap >= fg_threshold
    is_bg = trimap <= bg_threshold
    if is_bg.sum() == 0:
        raise ValueError(
            "Trimap did not contain background values (values <= %f)" % bg_threshold)
    if is_fg.sum() == 0:
        raise ValueError(
            "Trimap did not contain foreground values (values >= %f)" % fg_threshold)
    is_known = is_fg | is_bg
    is_unknown = ~is_known
    return is_fg, is_bg, is_known, is_unknown


def sanity_check_image(image):
    """Warn if ``image`` is not ``(?, ?, 3)``, not in [0, 1] or not float."""
    if len(image.shape) != 3 or image.shape[2] != 3:
        warnings.warn("Expected RGB image of shape (?, ?, 3), but image.shape is %s."
                      % str(image.shape), stacklevel=3)
    min_value = image.min()
    max_value = image.max()
    if min_value < 0.0:
        warnings.warn("Image values should be in [0, 1], but image.min() is %s." % min_value,
                      stacklevel=3)
    if max_value > 1.0:
        warnings.warn("Image values should be in [0, 1], but image.max() is %s." % max_value,
                      stacklevel=3)
    if image.dtype not in [np.float32, np.float64]:
        warnings.warn(
            "Unexpected image.dtype %s. Are you sure that you do not want to use np.float32 "
            "or np.float64 instead?" % image.dtype, stacklevel=3)
