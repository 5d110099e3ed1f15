"""Learned eddy-viscosity closure for 3-D LES (the 3-D counterpart of
TensorLBM's 2-D ``tensorlbm.ai`` closure: model.py, train.py, dataset.py,
inference.py, pipeline.py).  Every numeric step runs in libtlbm.so."""

from .dataset import filtered_moments, les_samples
from .inference import LearnedLESSolver
from .model import EddyViscosityMLP3D
from .train import TrainConfig, train_eddy_viscosity_model3d

__all__ = ["EddyViscosityMLP3D", "LearnedLESSolver", "TrainConfig", "filtered_moments", "les_samples",
           "train_eddy_viscosity_model3d"]
