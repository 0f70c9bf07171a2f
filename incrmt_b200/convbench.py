"""Timing of the tensor-core convolutions and of the U-Net built on them
(CUDA events, one GPU):

    python -m incrmt_b200.convbench                      # the layer table and the U-Net
    python -m incrmt_b200.convbench --shape 1,1024,1024,64,64 --reps 2 --variant 2

--shape B,H,W,Cin,Cout times one 3x3 layer (bias and ReLU); --variant pins
the kernel (incrmt_conv_set_variant: 0 automatic, 1 one tap per pipeline
stage, 2 row reuse, 3 row reuse with resident weights, 4 two 128-pixel halves
per CTA). Prints one JSON line
per layer or network: milliseconds per call and TFLOP/s of
2*9*Cin*Cout*pixels (the network: the sum over its layers).
"""
import argparse
import json
import sys

LAYERS = [(1, 1024, 1024, 64, 64), (1, 2048, 2048, 32, 32), (1, 1024, 1024, 32, 64), (1, 512, 512, 128, 128),
          (1, 256, 256, 256, 256), (1, 2048, 2048, 16, 32), (1, 2048, 2048, 96, 32), (1, 1024, 1024, 192, 64),
          (1, 512, 512, 384, 128)]


def unet_flops(H, W, base, levels=4):
    """Forward FLOPs of the library's U-Net (3x3 convolutions, 16 input
    channels, a 1x1 head of 16 outputs)."""
    C = [base << l for l in range(levels)]
    P = [H * W >> (2 * l) for l in range(levels)]
    f = 2 * 9 * 16 * C[0] * P[0] + 2 * 9 * C[0] * C[0] * P[0]
    for l in range(1, levels):
        f += 2 * 9 * C[l - 1] * C[l] * P[l] + 2 * 9 * C[l] * C[l] * P[l]
    for l in range(levels - 2, -1, -1):
        f += 2 * 9 * (C[l + 1] + C[l]) * C[l] * P[l] + 2 * 9 * C[l] * C[l] * P[l]
    return f + 2 * C[0] * 16 * P[0]


def time_layer(capi, torch, shape, reps):
    B, H, W, ci, co = shape
    dev = torch.device("cuda")
    x = torch.randn(B, H, W, ci, device=dev).to(torch.bfloat16)
    w = (torch.randn(9, co, ci, device=dev) * 0.05).to(torch.bfloat16)
    bias = torch.zeros(co, device=dev)
    y = torch.empty(B, H, W, co, device=dev, dtype=torch.bfloat16)

    def call():
        capi.conv_bf16(x.data_ptr(), B, H, W, ci, w.data_ptr(), 9, co, y.data_ptr(), bias.data_ptr(), True)

    for _ in range(3):
        call()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        call()
    e1.record()
    torch.cuda.synchronize()
    capi.conv_status()
    ms = e0.elapsed_time(e1) / reps
    return {"layer": list(shape), "ms": ms, "tflops": 2.0 * 9 * ci * co * B * H * W / ms / 1e9}


def time_unet(capi, torch, H, W, base, batch, reps):
    dev = torch.device("cuda")
    net = capi.UNet(4, base, seed=3)
    x = torch.randn(batch, H, W, 3, device=dev)
    y = torch.empty(batch, H, W, device=dev)
    for _ in range(3):
        net.forward(batch, H, W, x.data_ptr(), y.data_ptr())
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        net.forward(batch, H, W, x.data_ptr(), y.data_ptr())
    e1.record()
    torch.cuda.synchronize()
    capi.conv_status()
    ms = e0.elapsed_time(e1) / reps
    net.close()
    return {"unet": {"H": H, "W": W, "base": base, "batch": batch}, "forward_ms": ms,
            "tflops": unet_flops(H, W, base) * batch / ms / 1e9}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", default=None, help="B,H,W,Cin,Cout of one 3x3 layer")
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--variant", type=int, default=0)
    args = ap.parse_args(argv)
    import torch
    from incrmt_b200 import capi
    if not torch.cuda.is_available():
        sys.exit("convbench needs a GPU")
    capi.conv_set_variant(args.variant)
    try:
        shapes = [tuple(int(v) for v in args.shape.split(","))] if args.shape else LAYERS
        for sh in shapes:
            print(json.dumps({"variant": args.variant, **time_layer(capi, torch, sh, args.reps)}), flush=True)
        if not args.shape:
            print(json.dumps({"variant": args.variant, **time_unet(capi, torch, 2048, 2048, 32, 1, args.reps)}),
                  flush=True)
    finally:
        capi.conv_set_variant(0)


if __name__ == "__main__":
    main()
