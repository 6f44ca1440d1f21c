"""CPU restatement of the reference's SAP broadphase (rbc/BroadPhase.cpp,
rbc/BroadPhase.hpp), pure Python, for small object counts.

TEST INFRASTRUCTURE ONLY: the checker of the device broadphase in tests/.
The product never imports it.  It is pinned against the reference itself
(oracle/_ref, the reference compiled from its own sources) by
tests/test_oracle_cpu.py, and the device is checked against both.

The restatement keeps the reference's data and order exactly:
  * objects live in slots; removed slots go on a free list and are reused
    last-in first-out (broad_phase_insert, BroadPhase.cpp:169-197);
  * the endpoint list holds (float32 value, slot, is_max); insertion appends
    (min, max) (ep_insert, :21-47); removal drops the slot's endpoints in
    place (ep_remove, :50-56);
  * a move refits the fat AABB only when the tight AABB escapes it, with
    margin fat_margin + reinsert_threshold (broad_phase_move, :211-232);
  * update re-sorts with a stable insertion sort on the float value when
    anything changed (:80-94, :235-245), then sweeps in list order
    keeping an active list in opening order, emitting (min uid, max uid)
    for every 3-D fat-AABB overlap with the objects already open
    (bp_sweep, :104-152).
"""
import numpy as np


def _f32(x):
    """static_cast<float>(double), as a Python float holding the float32."""
    return float(np.float32(x))


def _overlap(a, b):
    # aabb_overlap (AABB.hpp:54-59), inclusive on every axis
    return (a[0] <= b[3] and a[3] >= b[0]) and (a[1] <= b[4] and a[4] >= b[1]) and \
           (a[2] <= b[5] and a[5] >= b[2])


def _contained(t, f):
    # aabb_contained (BroadPhase.cpp:8-13)
    return (t[0] >= f[0] and t[3] <= f[3] and t[1] >= f[1] and t[4] <= f[4] and
            t[2] >= f[2] and t[5] <= f[5])


def _expand(a, m):
    # aabb_expand (AABB.hpp:85-89)
    return [a[0] - m, a[1] - m, a[2] - m, a[3] + m, a[4] + m, a[5] + m]


class SapBroadPhase:
    def __init__(self, fat_margin=0.1, reinsert_threshold=0.05):
        self.fat_margin = fat_margin
        self.reinsert_threshold = reinsert_threshold
        self.objects = []      # dicts: tight, fat, uid, alive
        self.free_list = []
        self.endpoints = []    # [value, slot, is_max]
        self.pairs = []
        self.dirty = False

    def insert(self, user_id, tight):
        tight = [float(v) for v in tight]
        if self.free_list:
            slot = self.free_list.pop()
        else:
            slot = len(self.objects)
            self.objects.append(None)
        fat = _expand(tight, self.fat_margin)
        self.objects[slot] = {"tight": tight, "fat": fat, "uid": int(user_id), "alive": True}
        self.endpoints.append([_f32(fat[0]), slot, 0])
        self.endpoints.append([_f32(fat[3]), slot, 1])
        self.dirty = True
        return slot

    def remove(self, slot):
        self.objects[slot]["alive"] = False
        self.endpoints = [e for e in self.endpoints if e[1] != slot]
        self.free_list.append(slot)

    def move(self, slot, tight):
        o = self.objects[slot]
        tight = [float(v) for v in tight]
        o["tight"] = tight
        if _contained(tight, o["fat"]):
            return
        o["fat"] = _expand(tight, self.fat_margin + self.reinsert_threshold)
        for e in self.endpoints:
            if e[1] == slot:
                e[0] = _f32(o["fat"][3] if e[2] else o["fat"][0])
        self.dirty = True

    def move_swept(self, slot, tight, vel, dt):
        # broad_phase_move_swept (BroadPhase.hpp:228-249)
        m = self.fat_margin
        dv = [float(v) * dt for v in vel]
        emn = [m + (-d if d < 0 else 0.0) for d in dv]
        emx = [m + (d if d > 0 else 0.0) for d in dv]
        t = [tight[0] - emn[0], tight[1] - emn[1], tight[2] - emn[2],
             tight[3] + emx[0], tight[4] + emx[1], tight[5] + emx[2]]
        self.move(slot, t)

    def update(self):
        if self.dirty:
            ep = self.endpoints
            for i in range(1, len(ep)):
                key = ep[i]
                j = i - 1
                while j >= 0 and ep[j][0] > key[0]:
                    ep[j + 1] = ep[j]
                    j -= 1
                ep[j + 1] = key
            self.dirty = False
        self.pairs = []
        active = []
        for value, slot, is_max in self.endpoints:
            obj = self.objects[slot]
            if not obj["alive"]:
                continue
            if not is_max:
                for s2 in active:
                    other = self.objects[s2]
                    if not other["alive"] or not _overlap(obj["fat"], other["fat"]):
                        continue
                    a, b = obj["uid"], other["uid"]
                    self.pairs.append((a, b) if a < b else (b, a))
                active.append(slot)
            elif slot in active:
                active.remove(slot)
        return self.pairs

    def fat_aabb(self, slot):
        return list(self.objects[slot]["fat"])
