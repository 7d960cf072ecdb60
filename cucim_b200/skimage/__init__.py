"""Drop-in for the cucim.skimage functions on the separable filtering path:
filters.gaussian/sobel/prewitt/frangi, feature.hessian_matrix/
hessian_matrix_eigvals, color.rgb2gray and the img_as_float conversions."""

from . import color, feature, filters, util  # noqa: F401
