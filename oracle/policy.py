"""TEST INFRASTRUCTURE ONLY: the Depthmap frame policy replayed in Python.

Follows SeedMatrix::add_frames / need_add_reference / need_switchkeyframe /
extract_depth (seed_matrix.cu:106-209, 457-466) with float32 SE3 arithmetic
in the reference's operation order (se3.cuh:91-107, 179-195), so the slot
poses it produces are bit-identical to what the library computes.  Used to
drive the oracle over a frame sequence.
"""
import numpy as np

f32 = np.float32


def se3_identity():
    T = np.zeros(12, f32)
    T[0] = T[5] = T[10] = f32(1)
    return T


def se3_inv(a):
    a = np.asarray(a, f32)
    r = se3_identity()
    r[0], r[1], r[2] = a[0], a[4], a[8]
    r[4], r[5], r[6] = a[1], a[5], a[9]
    r[8], r[9], r[10] = a[2], a[6], a[10]
    r[3] = (-a[0] * a[3] - a[4] * a[7]) - a[8] * a[11]
    r[7] = (-a[1] * a[3] - a[5] * a[7]) - a[9] * a[11]
    r[11] = (-a[2] * a[3] - a[6] * a[7]) - a[10] * a[11]
    return r


def se3_mul(l, r):
    l = np.asarray(l, f32)
    r = np.asarray(r, f32)
    o = np.zeros(12, f32)
    for row in range(3):
        a = l[4 * row:4 * row + 4]
        for c in range(3):
            o[4 * row + c] = (a[0] * r[c] + a[1] * r[4 + c]) + a[2] * r[8 + c]
        o[4 * row + 3] = ((a[3] + a[0] * r[3]) + a[1] * r[7]) + a[2] * r[11]
    return o


def _moved(a_cw, b_cw, min_cos, max_base):
    a = se3_inv(a_cw)
    b = se3_inv(b_cw)
    z_cos = (a[2] * b[2] + a[6] * b[6]) + a[10] * b[10]
    d = np.array([a[3] - b[3], a[7] - b[7], a[11] - b[11]], f32)
    base = np.sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2])
    return float(z_cos) < min_cos or float(base) > max_base


class PolicyReplay:
    """Feeds frames; returns for each the outcome and, for dense frames, the
    slot frame indices (into the frames fed so far), slot poses and the fusion
    transform."""

    def __init__(self, num_slots=5, ratio=1, capacity=60):
        self.F = num_slots
        self.ratio = ratio
        self.capacity = capacity
        self.ring = []  # list of (frame id, T_frame_world), front first
        self.frame_index = 0
        self.initialized = False
        self.fuse_T = se3_identity()
        self.keyframe_T = se3_identity()
        self.keyframe_id = None

    def add(self, frame_id, T_curr_world):
        """Every outcome also carries the semi-dense step of the frame:
        sd_mode (1 first frame, 2 update, 3 update + keyframe switch),
        sd_key (frame id of the keyframe before the step) and sd_T
        (T_income<-key)."""
        T = np.asarray(T_curr_world, f32).reshape(12)
        self.frame_index += 1
        if not self.initialized:
            self.initialized = True
            self.keyframe_T = T
            self.keyframe_id = frame_id
            return dict(outcome="first", sd_mode=1, sd_key=None, sd_T=se3_identity())
        sd = dict(sd_mode=2, sd_key=self.keyframe_id, sd_T=se3_mul(T, se3_inv(self.keyframe_T)))
        if _moved(self.keyframe_T, T, 0.86, 0.5):
            self.keyframe_T = T
            self.keyframe_id = frame_id
            sd["sd_mode"] = 3
        if self.frame_index % self.ratio != 0:
            return dict(outcome="skip", **sd)
        out = dict(outcome="none", **sd)
        if len(self.ring) > 10:
            inv = se3_inv(T)
            slots, Ts = [], []
            for f in range(self.F):
                # (float)9 / 10.0 * (float)f is evaluated in double in C++
                k = min(int(9.0 / 10.0 * float(f)), len(self.ring) - 1)
                fid, Tf = self.ring[k]
                slots.append(fid)
                Ts.append(se3_mul(Tf, inv))
            out = dict(outcome="dense", slots=slots, T_slots=np.stack(Ts),
                       T_fuse=se3_mul(T, se3_inv(self.fuse_T)), **sd)
        if not self.ring or _moved(self.ring[0][1], T, 0.95, 0.03):
            self.ring.insert(0, (frame_id, T))
            if len(self.ring) > self.capacity:
                self.ring.pop()
        if out["outcome"] == "dense":
            self.fuse_T = T
        return out
