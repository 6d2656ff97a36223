"""fluide_engine_b200 -- B200-native hybrid particle-grid (PIC / FLIP / APIC) substep.

The compute path is the sm_100a library libfluide_b200.so (CUDA kernels + C ABI, include/fluide_b200.h);
this package binds it with ctypes and mirrors the reference's simulator API.
"""
from ._abi import (APIC, FLIP, PIC, AIR, FLUID, AUTO, CG, MGPCG, FluideError, kernel_launch_count, lib,  # noqa: F401
                   mesh_to_sdf, seed_regions, volume_field_vectors,
                   STAGE_SORT, STAGE_P2G, STAGE_MARK, STAGE_PRE, STAGE_DIFFUSE, STAGE_PRESSURE, STAGE_POST, STAGE_G2P,
                   STAGE_MOVE)
from .scene import Batch, Scene, Snapshot, face_shapes  # noqa: F401
from .simulators import (APICSimulator, BoundingBox3D, Collider, ColliderCollection, DirectionalField,  # noqa: F401
                         Emitter, ExternalForce, TriangleMeshCollider,
                         FLIPSimulator, Frame, HybridSimulator, OBJManager, PICSimulator, PointField, ScalarGrid3D,
                         SimulationRunner, SimulationStats, SwirlField, TriangleMesh, Vector3D, Vector3S,
                         VolumeEmitter, VolumeField)

__version__ = "0.1.0"
