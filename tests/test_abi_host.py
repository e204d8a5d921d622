"""Host-side checks that need no GPU: the C-ABI library loads, exports every
entry point include/hdrestir.h declares, its ctypes mirror has the C layout,
and argument errors come back as status codes with a message."""
import ctypes as C

import numpy as np
import pytest

from hdrestir_b200 import abi, configs

pytestmark = pytest.mark.skipif(not abi.LIB_PATH.exists(), reason="library not built")


def test_every_declared_symbol_is_exported():
    L = abi.lib()
    names = abi.exported_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_abi_version():
    assert abi.lib().hdr_abi_version() == 1


STRUCTS = {"hdr_mesh_desc": abi.MeshDesc, "hdr_instance_desc": abi.InstanceDesc,
           "hdr_material_desc": abi.MaterialDesc, "hdr_light_desc": abi.LightDesc, "hdr_scene_desc": abi.SceneDesc,
           "hdr_camera": abi.CameraDesc, "hdr_path_settings": abi.PathSettings, "hdr_ris_params": abi.RisParams,
           "hdr_ctx_desc": abi.CtxDesc}


def test_struct_layouts_match_the_c_header(tmp_path):
    """sizeof of every ABI struct as the C compiler lays it out from include/hdrestir.h."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "layout.c"
    body = "".join(f'printf("{n} %zu\\n", sizeof({n}));' for n in STRUCTS)
    body += 'printf("hdr_gbuffer_texel %zu\\n", sizeof(hdr_gbuffer_texel));'
    src.write_text(f'#include <stdio.h>\n#include "hdrestir.h"\nint main(void){{{body}return 0;}}\n')
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", str(abi.LIB_PATH.parent.parent / "include"), str(src), "-o", str(exe)], check=True)
    sizes = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                         check=True).stdout.splitlines())
    for name, cls in STRUCTS.items():
        assert C.sizeof(cls) == int(sizes[name]), name
    assert abi.GBUFFER_DTYPE.itemsize == int(sizes["hdr_gbuffer_texel"])


def test_null_arguments_fail_cleanly():
    L = abi.lib()
    assert L.hdr_ctx_create(None, None) == abi.HDR_EINVAL
    assert b"NULL" in L.hdr_last_error() or L.hdr_last_error()
    assert L.hdr_scene_upload(None, None) == abi.HDR_EINVAL
    assert L.hdr_raycast(None, None, 0, 0) == abi.HDR_EINVAL
    assert L.hdr_accumulate(None, 0, 1, 0) == abi.HDR_EINVAL
    with pytest.raises(abi.HdrError):
        abi.check(abi.HDR_EINVAL)


def test_scene_desc_round_trip():
    sc, cam = configs.config0(16, 16)
    d = sc.c_desc()
    assert d.num_meshes == 12 and d.num_instances == 12 and d.num_lights == 2
    assert d.meshes[0].num_triangles == 2
    np.testing.assert_allclose(np.ctypeslib.as_array(d.instances[3].transform), np.eye(4).reshape(-1))
    cd = cam.c_desc()
    assert cd.width == 16 and cd.has_params == 0
