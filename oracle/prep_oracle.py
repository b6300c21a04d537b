"""numpy restatement of the reference's RTM input preprocessing
(run/generate_input_data.py:28-46) -- TEST INFRASTRUCTURE ONLY: checks
fwi_prepare_rtm_input.  Same dtypes as the script: FP32 data and offsets, a
truncated FP32 direct-wave sample, an FP64 taper."""
import numpy as np


def rtm_input(data_nt_nr, sx, sy, rec_xy, dt, velocity=3600, time_delay=0.18, gstd=30):
    data = np.array(data_nt_nr, dtype=np.float32, copy=True)       # (nt, nrec)
    nt = data.shape[0]
    data *= np.float32(1.0 / np.float64(np.max(np.abs(data))))
    rx = np.asarray(rec_xy[:, 0], np.float32)
    ry = np.asarray(rec_xy[:, 1], np.float32)
    distance = np.sqrt((rx - np.float32(sx)) ** 2 + (ry - np.float32(sy)) ** 2)
    tId = np.array((distance / np.float32(velocity) + np.float32(time_delay)) / np.float32(dt), dtype=int)
    timeId = np.arange(nt)
    for r in range(data.shape[1]):
        taper = np.exp(-0.5 * ((timeId - tId[r]) / gstd) ** 2)[:tId[r]]
        data[:tId[r], r] = (data[:tId[r], r].astype(np.float64) * taper).astype(np.float32)
    return data
