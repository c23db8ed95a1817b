"""``cutout`` and the image-file helpers it uses.

Drop-ins for ``cutout(image_path, trimap_path, cutout_path)``
(pymatting/cutout/cutout.py:6-36) and for ``load_image``, ``save_image``,
``stack_images`` and ``blend`` (pymatting/util/util.py:213-290, 581-643).
Files are decoded and encoded by PIL on the host, as in the reference; the
two compute steps in between run on the device: ``estimate_alpha_cf``
(closed-form alpha) and ``estimate_foreground_ml`` (foreground colours in
the reference's sweep order). PIL is needed only for the file helpers.
"""

import os

import numpy as np

from .alpha import estimate_alpha_cf
from .foreground import estimate_foreground_ml

__all__ = ["cutout", "load_image", "save_image", "stack_images", "blend"]

_FILTERS = ("bicubic", "bilinear", "box", "hamming", "lanczos", "nearest", "none")


def _pil():
    try:
        from PIL import Image
    except ImportError as e:   # pragma: no cover - PIL is in the image
        raise ImportError("the image-file helpers of pymatting_b200 need Pillow") from e
    return Image


def _resize_pil_image(image, size, resample="bicubic"):
    Image = _pil()
    filters = {"bicubic": Image.BICUBIC, "bilinear": Image.BILINEAR, "box": Image.BOX,
               "hamming": Image.HAMMING, "lanczos": Image.LANCZOS, "nearest": Image.NEAREST,
               "none": Image.NEAREST}
    if not hasattr(size, "__iter__"):
        size = (int(image.width * size), int(image.height * size))
    return image.resize(size, filters[resample.lower()])


def load_image(path, mode=None, size=None, resample="box"):
    """Load an image file as a float64 array in [0, 1]. ``mode`` is "GRAY",
    "RGB" or another PIL mode; ``size`` a scale factor or a (width, height)
    pair, resized with ``resample``."""
    Image = _pil()
    image = Image.open(path)
    if mode is not None:
        mode = mode.upper()
        mode = "L" if mode == "GRAY" else mode
        image = image.convert(mode)
    if size is not None:
        image = _resize_pil_image(image, size, resample)
    return np.array(image) / 255.0


def save_image(path, image, make_directory=True):
    """Save a uint8 image, or a float image in [0, 1] (scaled by 255,
    clipped and truncated to uint8)."""
    assert image.dtype in [np.uint8, np.float32, np.float64]
    if image.dtype in [np.float32, np.float64]:
        image = np.clip(image * 255, 0, 255).astype(np.uint8)
    if make_directory:
        directory, _ = os.path.split(path)
        if len(directory) > 0:
            os.makedirs(directory, exist_ok=True)
    _pil().fromarray(image).save(path)


def stack_images(*images):
    """Concatenate images along the channel axis (2-D images count as one
    channel)."""
    images = [(image if len(image.shape) == 3 else image[:, :, np.newaxis]) for image in images]
    return np.concatenate(images, axis=2)


def blend(foreground, background, alpha):
    """Compose alpha * foreground + (1 - alpha) * background."""
    if len(alpha.shape) == 2:
        alpha = alpha[:, :, np.newaxis]
    return alpha * foreground + (1 - alpha) * background


def cutout(image_path, trimap_path, cutout_path):
    """Write the RGBA cutout of an image: closed-form alpha from the trimap,
    foreground colours by multi-level estimation, stacked and saved."""
    image = load_image(image_path, "RGB")
    trimap = load_image(trimap_path, "GRAY")
    if image.shape[:2] != trimap.shape[:2]:
        raise ValueError("Input image and trimap must have same size")
    alpha = estimate_alpha_cf(image, trimap)
    foreground = estimate_foreground_ml(image, alpha)
    save_image(cutout_path, stack_images(foreground, alpha))
