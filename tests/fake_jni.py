"""A fake JNIEnv for driving the JNI entry point without a JVM.

The function table has the JNI specification's layout (233 slots; the slots
the entry point uses are filled, see include/readdy_b200_jni_types.h).  Java
objects are integer handles into a Python dict: strings, float arrays and the
TopGPU object whose frameCallback and cReactions field a test scripts.
"""
import ctypes as C

import numpy as np

SLOTS = {"DeleteLocalRef": 23, "GetObjectClass": 31, "GetMethodID": 33, "CallBooleanMethodA": 39,
         "GetFieldID": 94, "GetObjectField": 95, "GetStringUTFChars": 169, "ReleaseStringUTFChars": 170,
         "GetArrayLength": 171, "NewFloatArray": 181, "GetPrimitiveArrayCritical": 222,
         "ReleasePrimitiveArrayCritical": 223, "ExceptionCheck": 228}
TABLE = 233

VP = C.c_void_p
CP = C.c_char_p


class _Env(C.Structure):
    _fields_ = [("functions", C.POINTER(VP * TABLE))]


class FakeJVM:
    """frame_callback(frame, positions float32 array) -> bool;
    reactions(frame) -> float list for the cReactions field (or None)."""

    METHOD = 0x5151
    FIELD = 0x6161
    CLASS = 0x7171

    def __init__(self, frame_callback, reactions=None):
        self.frame_callback = frame_callback
        self.reactions = reactions
        self.objs = {}
        self.next = 0x1000
        self.calls = []
        self.frame = -1
        self.keep = []
        self.table = (VP * TABLE)()
        self._install()
        self.env = _Env(C.pointer(self.table))

    def handle(self, obj):
        h = self.next
        self.next += 8
        self.objs[h] = obj
        return h

    def jstring(self, s):
        return self.handle(C.create_string_buffer(s.encode()))

    def _fn(self, name, restype, *args):
        def deco(f):
            def wrapped(*a):
                self.calls.append(name)
                return f(*a)
            cb = C.CFUNCTYPE(restype, *args)(wrapped)
            self.keep.append(cb)
            self.table[SLOTS[name]] = C.cast(cb, VP)
            return f
        return deco

    def _install(self):
        unexpected = C.CFUNCTYPE(None)(lambda: self.calls.append("UNEXPECTED"))
        self.keep.append(unexpected)
        for i in range(TABLE):
            self.table[i] = C.cast(unexpected, VP)

        @self._fn("DeleteLocalRef", None, VP, VP)
        def _del(env, o):
            self.objs.pop(o, None)

        @self._fn("GetObjectClass", VP, VP, VP)
        def _cls(env, o):
            return self.CLASS

        @self._fn("GetMethodID", VP, VP, VP, CP, CP)
        def _mid(env, c, name, sig):
            return self.METHOD if (name == b"frameCallback" and sig == b"(I[F)Z") else None

        @self._fn("CallBooleanMethodA", C.c_uint8, VP, VP, VP, C.POINTER(C.c_uint64))
        def _call(env, o, mid, args):
            frame = C.c_int32(args[0] & 0xffffffff).value
            arr = self.objs[args[1]]
            self.frame = frame
            return 1 if self.frame_callback(frame, arr.copy()) else 0

        @self._fn("GetFieldID", VP, VP, VP, CP, CP)
        def _fid(env, c, name, sig):
            return self.FIELD if (name == b"cReactions" and sig == b"[F") else None

        @self._fn("GetObjectField", VP, VP, VP, VP)
        def _getf(env, o, f):
            r = self.reactions(self.frame) if self.reactions else None
            if r is None:
                return None
            return self.handle(np.asarray(r, dtype=np.float32))

        @self._fn("GetStringUTFChars", VP, VP, VP, VP)
        def _utf(env, s, iscopy):
            return C.cast(self.objs[s], VP).value

        @self._fn("ReleaseStringUTFChars", None, VP, VP, VP)
        def _rel(env, s, p):
            pass

        @self._fn("GetArrayLength", C.c_int32, VP, VP)
        def _len(env, a):
            return int(self.objs[a].size)

        @self._fn("NewFloatArray", VP, VP, C.c_int32)
        def _new(env, n):
            return self.handle(np.zeros(n, np.float32))

        @self._fn("GetPrimitiveArrayCritical", VP, VP, VP, VP)
        def _crit(env, a, iscopy):
            return self.objs[a].ctypes.data

        @self._fn("ReleasePrimitiveArrayCritical", None, VP, VP, VP, C.c_int32)
        def _relc(env, a, p, mode):
            pass

        @self._fn("ExceptionCheck", C.c_uint8, VP)
        def _exc(env):
            return 0

    def run(self, lib, paths, testmode=False):
        f = lib.Java_readdy_impl_sim_top_TopGPU_cCreateSimulation
        f.restype = None
        f.argtypes = [C.POINTER(_Env), VP, C.c_uint8] + [VP] * 6
        obj = self.handle("TopGPU")
        js = [self.jstring(paths[k]) for k in ("param_particles", "tplgy_potentials", "param_groups",
                                                "tplgy_coordinates", "tplgy_groups", "param_global")]
        f(C.byref(self.env), obj, int(testmode), *js)


def write_inputs(d, n=400, frames=3, seed=1, L=40.0, dimers=0):
    """ReaDDy input files (param_particles, tplgy_potentials, param_global,
    tplgy_coordinates, param_groups, tplgy_groups) for a 2-species system in
    a periodic box with a CUBE wall and harmonic repulsion; the first
    2 x dimers particles form spring-bonded dimer groups."""
    rng = np.random.default_rng(seed)
    p = {k: str(d / f"{k}.xml") for k in ("param_particles", "tplgy_potentials", "param_groups",
                                          "tplgy_coordinates", "tplgy_groups", "param_global")}
    open(p["param_particles"], "w").write("""<?xml version="1.0" encoding="UTF-8"?>
<!-- two species -->
<param_particles version="1.1">
 <particle><type>A</type><diffusionConstant>1e+6</diffusionConstant>
  <numberOfDummyParticles>0</numberOfDummyParticles>
  <collisionRadiusMap><collisionRadius><partnerType>default</partnerType><radius>1.5</radius></collisionRadius>
  </collisionRadiusMap>
  <reactionRadiusMap><reactionRadius><partnerType>default</partnerType><radius>1.5</radius></reactionRadius></reactionRadiusMap>
 </particle>
 <particle><type>B</type><diffusionConstant>0.5e+6</diffusionConstant>
  <collisionRadiusMap><collisionRadius><partnerType>default</partnerType><radius>2</radius></collisionRadius>
   <collisionRadius><partnerType>A</partnerType><radius>1.75</radius></collisionRadius></collisionRadiusMap>
 </particle>
</param_particles>
""")
    h = L / 2 - 2
    open(p["tplgy_potentials"], "w").write(f"""<tplgy_potentials version="1.1">
 <pot name="wall" type="CUBE" subtype="attractive" forceConst="10" origin="[{-h},{-h},{-h}]"
      extension="[{2 * h},{2 * h},{2 * h}]" considerParticleRadius="true" affectedParticleTypeIds="all"
      affectedParticleIds="" />
 <pot name="rep" type="HARMONIC" subtype="repulsive" forceConst="10" affectedParticleTypeIdPairs="all"
      affectedParticleIdPairs="" />
 <pot name="weak" type="WEAK_INTERACTION_PIECEWISE_HARMONIC" forceConst="10" depth="2" length="1.3"
      affectedParticleTypeIdPairs="[[0,1]]" affectedParticleIdPairs="" />
</tplgy_potentials>
""")
    open(p["param_global"], "w").write(f"""<param_global version="1.1">
 <nSimulationSteps>{frames}</nSimulationSteps>
 <dt>1e-7</dt>
 <dtOpenMM>1e-9</dtOpenMM>
 <cudaDeviceIndex>0</cudaDeviceIndex>
 <T>293.15</T>
 <Kb>0.0083144621</Kb>
 <latticeBounds>[[{-L / 2},{L / 2}];[{-L / 2},{L / 2}];[{-L / 2},{L / 2}]]</latticeBounds>
</param_global>
""")
    xyz = rng.uniform(-h + 1, h - 1, size=(n, 3))
    types = rng.integers(0, 2, n)
    for g in range(dimers):   # partner 3 nm away along x
        xyz[2 * g + 1] = xyz[2 * g] + [3.0, 0.0, 0.0]
        types[2 * g] = types[2 * g + 1] = 0
    lines = ['<tplgy_coords version="1.1" stepId="0">']
    for i in range(n):
        lines.append(f'<p id="{1000 + i}" type="{types[i]}" c="{float(xyz[i, 0])!r},{float(xyz[i, 1])!r},{float(xyz[i, 2])!r}"/>')
    lines.append("</tplgy_coords>")
    open(p["tplgy_coordinates"], "w").write("\n".join(lines) + "\n")
    if dimers:
        open(p["param_groups"], "w").write("""<param_groups version="1.1">
 <particleGroup>
  <type>dimer</type>
  <templateOrigin>[0.0,0.0,0.0]</templateOrigin>
  <templateNormal>[0,0,1]</templateNormal>
  <buildingBlocks>
   <particle internalId="0" type="A" templateC="[0.0,0.0,0.0]"/>
   <particle internalId="1" type="A" templateC="[3.0,0.0,0.0]"/>
  </buildingBlocks>
  <potentials>
   <pot name="spring" type="HARMONIC" subtype="spring" forceConst="20.0" affectedInternalIdPairs="[[0,1]]"/>
   <pot name="stiff" type="StiffnessInteraction" forceConst="3" affectedInternalIdPairs="[[0,1]]"/>
  </potentials>
  <maxNumberOfGroupAssignmentsPerParticle>1</maxNumberOfGroupAssignmentsPerParticle>
 </particleGroup>
</param_groups>
""")
        g = ['<tplgy_groups version="1.1">']
        for i in range(dimers):
            g.append(f'<g id="{i}" type="0" internalAndParticleId="[[0,{1000 + 2 * i}];[1,{1001 + 2 * i}]]"/>')
        g.append("</tplgy_groups>")
        open(p["tplgy_groups"], "w").write("\n".join(g) + "\n")
    else:
        open(p["param_groups"], "w").write('<param_groups version="1.1"></param_groups>\n')
        open(p["tplgy_groups"], "w").write('<tplgy_groups version="1.1"></tplgy_groups>\n')
    return p, xyz, types
