"""B200-native BIMP keypoint detector (sm_100a), Python side of the C ABI."""
from .api import (KP_MAX_POINTS, Batch, Context, CudaStuff, KeyPoint, default_params, detect_host,
                  downloadKeypoints, getKeypoints, keypoint_matrix_to_records, makeLambdasLin,
                  makeLambdasLog, snapTransformSize, uploadKeypoints)

__all__ = ["KP_MAX_POINTS", "Batch", "Context", "CudaStuff", "KeyPoint", "default_params", "detect_host",
           "downloadKeypoints", "getKeypoints", "keypoint_matrix_to_records", "makeLambdasLin",
           "makeLambdasLog", "snapTransformSize", "uploadKeypoints"]
