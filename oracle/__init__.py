"""ORACLE -- test infrastructure only: the CPU restatement of the reference
kernels and the harness around the reference's own CUDA build. The product
(ip_cu_lbm_b200) never imports this package."""
