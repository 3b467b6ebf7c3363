"""Host logic of bench.py that needs no GPU: the DRAM traffic table under profiles/ and the
naming of the local kernel the autotuner chose."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_traffic_table_has_the_local_kernels():
    b = load_bench()
    assert b.read_traffic("local_pencil_kernel_f32") == 65234
    assert b.read_traffic("local_fused_pf_kernel_f32") == 70326
    assert b.read_traffic("no_such_kernel") is None


def test_local_kernel_named_from_the_autotuner_choice():
    b = load_bench()
    line = ["chosen: projector chunk 32, addition 8 blocks per CTA, local %s, CUDA-core projector"]
    name, key = b.local_kernel_of([line[0] % "pencils"])
    assert name.startswith("local_pencil_kernel") and key == "local_pencil_kernel_f32"
    name, key = b.local_kernel_of([line[0] % "rows with loads ahead"])
    assert name.startswith("local_fused_pf_kernel") and key == "local_fused_pf_kernel_f32"
    name, key = b.local_kernel_of([line[0] % "plain rows"])
    assert name.startswith("local_fused_kernel") and key is None
