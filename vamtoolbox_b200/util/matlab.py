"""vamtoolbox.util.matlab (vamtoolbox/util/matlab.py:6-63): results to a MATLAB .mat file."""
from scipy import io

from .. import geometry


def saveMatData(filepath, target_geo=None, sinogram=None, reconstruction=None):
    """Save the arrays of a Sinogram ('opt_proj'), a Reconstruction ('opt_recon') and a TargetGeometry
    ('target') to filepath (.mat); an argument of any other type raises, as in the reference."""
    save = {}
    for key, obj, cls, what in (("opt_proj", sinogram, geometry.Sinogram, "sinogram argument must be of type "
                                 "geometry.Sinogram"),
                                ("opt_recon", reconstruction, geometry.Reconstruction, "reconstruction argument must "
                                 "be of type geometry.Reconstruction"),
                                ("target", target_geo, geometry.TargetGeometry, "target_geo argument must be of type "
                                 "geometry.TargetGeometry")):
        if isinstance(obj, cls):
            save[key] = obj.array
        elif obj is not None:
            raise Exception(what)
    io.savemat(filepath, save)
