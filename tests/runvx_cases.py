"""Graph cases for the runvx parity loop: one per in-scope GDF test of the reference
(tests/amd_openvx_gdfs/<group>/<name>.gdf, named in each case), written out here as GDF text
with seeded random input frames instead of the reference's uniform images, so that every
output pixel depends on the input.

Each case gives the data and node statements of its graph; `gdf(case, tmp, mode)` writes the
text for one runvx run: mode "write" saves every output image and keypoint array (the
reference run), mode "compare" checks every output against those files with runvx's own
compare facilities (utilities/runvx/vxImage.cpp:599 inside the rectangle the reference
defines -- a stencil's border is undefined in OpenVX with border mode UNDEFINED --, and
utilities/runvx/vxArray.cpp:462 for keypoints: coordinates exact, strengths within 1e-10)."""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

# bytes per pixel of each plane (plane width divisor, plane height divisor, bytes per pixel)
_PLANES = {
    "U008": [(1, 1, 1)], "S016": [(1, 1, 2)], "U016": [(1, 1, 2)], "U032": [(1, 1, 4)], "S032": [(1, 1, 4)],
    "RGB2": [(1, 1, 3)], "RGBA": [(1, 1, 4)], "RGBX": [(1, 1, 4)], "YUYV": [(1, 1, 2)], "UYVY": [(1, 1, 2)],
    "NV12": [(1, 1, 1), (2, 2, 2)], "NV21": [(1, 1, 1), (2, 2, 2)], "IYUV": [(1, 1, 1), (2, 2, 1), (2, 2, 1)],
    "YUV4": [(1, 1, 1), (1, 1, 1), (1, 1, 1)],
}


def frame_bytes(w, h, fmt):
    return sum(((w + dx - 1) // dx) * ((h + dy - 1) // dy) * b for dx, dy, b in _PLANES[fmt])


@dataclass
class Case:
    name: str                      # the reference GDF this case mirrors (<group>/<name>.gdf)
    inputs: list                   # (data name, W, H, format)
    outputs: list                  # (data name, W, H, format, margin)
    lines: list = field(default_factory=list)    # other data statements
    node: str = ""
    arrays: list = field(default_factory=list)   # keypoint array outputs: (data name, capacity)


def _unary(name, kernel, fmt_in, fmt_out, margin=0, extra="", w=1920, h=1080, ow=None, oh=None, lines=()):
    return Case(name, [("input_1", w, h, fmt_in)], [("output_1", ow or w, oh or h, fmt_out, margin)], list(lines),
                f"node org.khronos.openvx.{kernel} input_1 output_1{extra}")


def _binary(name, kernel, f1, f2, fo, mid=""):
    return Case(name, [("input_1", 1920, 1080, f1), ("input_2", 1920, 1080, f2)], [("output_1", 1920, 1080, fo, 0)], [],
                f"node org.khronos.openvx.{kernel} input_1 input_2{mid} output_1")


CASES = [
    # filter/
    _unary("filter/Box_U8_U8_3x3", "box_3x3", "U008", "U008", 1),
    _unary("filter/Dilate_U8_U8_3x3", "dilate_3x3", "U008", "U008", 1),
    _unary("filter/Erode_U8_U8_3x3", "erode_3x3", "U008", "U008", 1),
    _unary("filter/Gaussian_U8_U8_3x3", "gaussian_3x3", "U008", "U008", 1),
    _unary("filter/Median_U8_U8_3x3", "median_3x3", "U008", "U008", 1),
    Case("filter/ScaleGaussianHalf_U8_U8_5x5", [("input_1", 1920, 1080, "U008")], [("output_1", 960, 540, "U008", 1)],
         ["data scalar = scalar:INT32,5"], "node org.khronos.openvx.halfscale_gaussian input_1 output_1 scalar"),
    Case("filter/Sobel_S16S16_U8_3x3_GXY", [("input_1", 1920, 1080, "U008")],
         [("output_1", 1920, 1080, "S016", 1), ("output_2", 1920, 1080, "S016", 1)], [],
         "node org.khronos.openvx.sobel_3x3 input_1 output_1 output_2"),
    _unary("filter/Sobel_S16_U8_3x3_GX", "sobel_3x3", "U008", "S016", 1, " null"),
    Case("filter/Sobel_S16_U8_3x3_GY", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "S016", 1)], [],
         "node org.khronos.openvx.sobel_3x3 input_1 null output_1"),
    Case("filter/Convolve_U8_U8_3x3", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "U008", 1)],
         ["data input_matrix = convolution:3,3:INIT,{-1;-1;-1;-1;16;-1;-1;-1;-1}"],
         "node org.khronos.openvx.custom_convolution input_1 input_matrix output_1"),
    Case("filter/Convolve_S16_U8_3x3", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "S016", 1)],
         ["data input_matrix = convolution:3,3:INIT,{1;2;1;0;0;0;-1;-2;-1}"],
         "node org.khronos.openvx.custom_convolution input_1 input_matrix output_1"),
    Case("filter/Convolve_U8_U8_9x3", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "U008", 4)],
         ["data input_matrix = convolution:9,3:INIT,{" + ";".join(str((7 * i) % 11 - 5) for i in range(27)) + "}"],
         "node org.khronos.openvx.custom_convolution input_1 input_matrix output_1"),
    Case("filter/Convolve_S16_U8_9x3", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "S016", 4)],
         ["data input_matrix = convolution:9,3:INIT,{" + ";".join(str((13 * i) % 17 - 8) for i in range(27)) + "}"],
         "node org.khronos.openvx.custom_convolution input_1 input_matrix output_1"),
    # color/
    Case("color/ChannelCombine_U16_U8U8", [("input_1", 960, 540, "U008"), ("input_2", 960, 540, "U008")],
         [("output_1", 1920, 1080, "NV12", 0)], ["data luma = image:1920,1080,U008"],
         "node org.khronos.openvx.channel_combine luma input_1 input_2 null output_1"),
    Case("color/ChannelCombine_U24_U8U8U8_RGB", [("input_1", 1920, 1080, "U008"), ("input_2", 1920, 1080, "U008"),
                                                ("input_3", 1920, 1080, "U008")], [("output_1", 1920, 1080, "RGB2", 0)], [],
         "node org.khronos.openvx.channel_combine input_1 input_2 input_3 null output_1"),
    Case("color/ChannelCombine_U32_U8U8U8U8_RGBX", [("input_%d" % i, 1920, 1080, "U008") for i in (1, 2, 3, 4)],
         [("output_1", 1920, 1080, "RGBA", 0)], [],
         "node org.khronos.openvx.channel_combine input_1 input_2 input_3 input_4 output_1"),
    Case("color/ChannelCombine_U32_U8U8U8_UYVY", [("input_1", 1920, 1080, "U008"), ("input_2", 960, 1080, "U008"),
                                                 ("input_3", 960, 1080, "U008")], [("output_1", 1920, 1080, "UYVY", 0)], [],
         "node org.khronos.openvx.channel_combine input_1 input_2 input_3 null output_1"),
    Case("color/ChannelCombine_U32_U8U8U8_YUYV", [("input_1", 1920, 1080, "U008"), ("input_2", 960, 1080, "U008"),
                                                 ("input_3", 960, 1080, "U008")], [("output_1", 1920, 1080, "YUYV", 0)], [],
         "node org.khronos.openvx.channel_combine input_1 input_2 input_3 null output_1"),
    Case("color/ChannelExtract_U8_U16_Pos0", [("input_1", 1920, 1080, "YUYV")], [("output_1", 1920, 1080, "U008", 0)], [],
         "node org.khronos.openvx.channel_extract input_1 !CHANNEL_Y output_1"),
    Case("color/ChannelExtract_U8_U24_Pos1", [("input_1", 1920, 1080, "RGB2")], [("output_1", 1920, 1080, "U008", 0)], [],
         "node org.khronos.openvx.channel_extract input_1 !CHANNEL_G output_1"),
    Case("color/ChannelExtract_U8_U32_Pos3", [("input_1", 1920, 1080, "RGBA")], [("output_1", 1920, 1080, "U008", 0)], [],
         "node org.khronos.openvx.channel_extract input_1 !CHANNEL_A output_1"),
    _unary("color/ColorConvert_IYUV_RGB", "color_convert", "RGB2", "IYUV"),
    _unary("color/ColorConvert_NV12_RGB", "color_convert", "RGB2", "NV12"),
    Case("color/ColorDepth_S16_U8", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "S016", 0)],
         ["data scalar = scalar:INT32,1"], "node org.khronos.openvx.convertdepth input_1 output_1 !WRAP scalar"),
    Case("color/ColorDepth_U8_S16_Sat", [("input_1", 1920, 1080, "S016")], [("output_1", 1920, 1080, "U008", 0)],
         ["data scalar = scalar:INT32,1"], "node org.khronos.openvx.convertdepth input_1 output_1 !SATURATE scalar"),
    Case("color/ColorDepth_U8_S16_Wrap", [("input_1", 1920, 1080, "S016")], [("output_1", 1920, 1080, "U008", 0)],
         ["data scalar = scalar:INT32,1"], "node org.khronos.openvx.convertdepth input_1 output_1 !WRAP scalar"),
    # geometric/
    _unary("geometric/ScaleImage_U8_U8_Area", "scale_image", "U008", "U008", 0, " !AREA", ow=960, oh=540),
    _unary("geometric/ScaleImage_U8_U8_Bilinear", "scale_image", "U008", "U008", 0, " !BILINEAR", ow=960, oh=540),
    _unary("geometric/ScaleImage_U8_U8_Nearest", "scale_image", "U008", "U008", 0, " !NEAREST_NEIGHBOR", ow=960, oh=540),
    Case("geometric/WarpAffine_U8_U8_Bilinear_Constant", [("input_1", 1920, 1080, "U008")],
         [("output_1", 1920, 1080, "U008", 0)], ["data affine_matrix = matrix:FLOAT32,2,3:INIT,{0.25;0;0;0.5;20;20}"],
         "node org.khronos.openvx.warp_affine input_1 affine_matrix !BILINEAR output_1 attr:BORDER_MODE:CONSTANT,0"),
    Case("geometric/WarpAffine_U8_U8_Nearest_Constant", [("input_1", 1920, 1080, "U008")],
         [("output_1", 1920, 1080, "U008", 0)], ["data affine_matrix = matrix:FLOAT32,2,3:INIT,{0.25;0;0;0.5;20;20}"],
         "node org.khronos.openvx.warp_affine input_1 affine_matrix !NEAREST_NEIGHBOR output_1 attr:BORDER_MODE:CONSTANT,0"),
    Case("geometric/WarpPerspective_U8_U8_Nearest_Constant", [("input_1", 1920, 1080, "U008")],
         [("output_1", 1920, 1080, "U008", 0)],
         ["data perspective_matrix = matrix:FLOAT32,3,3:INIT,{2;0.1;0;2;1.9;0;-1200;-360;1}"],
         "node org.khronos.openvx.warp_perspective input_1 perspective_matrix !NEAREST_NEIGHBOR output_1 "
         "attr:BORDER_MODE:CONSTANT,0"),
    Case("geometric/WarpPerspective_U8_U8_Bilinear_Constant", [("input_1", 1920, 1080, "U008")],
         [("output_1", 1920, 1080, "U008", 0)],
         ["data perspective_matrix = matrix:FLOAT32,3,3:INIT,{2;0.1;0;2;1.9;0;-1200;-360;1}"],
         "node org.khronos.openvx.warp_perspective input_1 perspective_matrix !BILINEAR output_1 "
         "attr:BORDER_MODE:CONSTANT,0"),
    # arithmetic/
    _binary("arithmetic/AbsDiff_U8_U8U8", "absdiff", "U008", "U008", "U008"),
    _binary("arithmetic/AbsDiff_S16_S16S16_Sat", "absdiff", "S016", "S016", "S016"),
    _binary("arithmetic/Add_U8_U8U8_Wrap", "add", "U008", "U008", "U008", " !WRAP"),
    _binary("arithmetic/Add_U8_U8U8_Sat", "add", "U008", "U008", "U008", " !SATURATE"),
    _binary("arithmetic/Add_S16_U8U8_Wrap", "add", "U008", "U008", "S016", " !WRAP"),
    _binary("arithmetic/Add_S16_S16U8_Sat", "add", "S016", "U008", "S016", " !SATURATE"),
    _binary("arithmetic/Add_S16_S16S16_Wrap", "add", "S016", "S016", "S016", " !WRAP"),
    _binary("arithmetic/Sub_U8_U8U8_Sat", "subtract", "U008", "U008", "U008", " !SATURATE"),
    _binary("arithmetic/Sub_S16_U8S16_Sat", "subtract", "U008", "S016", "S016", " !SATURATE"),
    _binary("arithmetic/Sub_S16_S16S16_Wrap", "subtract", "S016", "S016", "S016", " !WRAP"),
    _binary("arithmetic/Magnitude_S16_S16S16", "magnitude", "S016", "S016", "S016"),
    # logical/
    _binary("logical/And_U8_U8U8", "and", "U008", "U008", "U008"),
    _binary("logical/Or_U8_U8U8", "or", "U008", "U008", "U008"),
    _binary("logical/Xor_U8_U8U8", "xor", "U008", "U008", "U008"),
    _unary("logical/Not_U8_U8", "not", "U008", "U008"),
    # statistical/
    Case("statistical/Threshold_U8_U8_Binary", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "U008", 0)],
         ["data binary_threshold = threshold:BINARY,U008,U008:INIT,127"],
         "node org.khronos.openvx.threshold input_1 binary_threshold output_1"),
    Case("statistical/Threshold_U8_U8_Range", [("input_1", 1920, 1080, "U008")], [("output_1", 1920, 1080, "U008", 0)],
         ["data range_threshold = threshold:RANGE,U008,U008:INIT,100,200"],
         "node org.khronos.openvx.threshold input_1 range_threshold output_1"),
]

# vision/: Canny with each gradient size and norm, on a luma plane extracted from IYUV as the
# reference's GDFs do (they read a 1280x720 clip; here a seeded random frame)
for gs in (3, 5, 7):
    for norm in ("L1", "L2"):
        CASES.append(Case(
            f"vision/Canny_{gs}x{gs}_{norm}NORM", [("input_iyuv", 1280, 720, "IYUV")],
            [("output_1", 1280, 720, "U008", gs // 2 + 1)],
            ["data inter_luma = image:1280,720,U008", "data input_hyst = threshold:RANGE,U008,U008:INIT,80,100",
             f"data input_gradient_size = scalar:INT32,{gs}"],
            "node org.khronos.openvx.channel_extract input_iyuv !CHANNEL_Y inter_luma\n"
            f"node org.khronos.openvx.canny_edge_detector inter_luma input_hyst input_gradient_size !NORM_{norm} output_1"))


# vision/: Harris at each gradient / block size and FAST with and without suppression, on a
# seeded random 1280x720 frame (W % 16 == 0: the gradient and circle reads across row ends
# reach the neighbouring rows); every corner of the list is compared
for gs, tc in ((3, 1e-4), (5, 1e-3), (7, 1e-3)):
    CASES.append(Case(
        f"vision/Harris_{gs}x{gs}", [("input_1", 1280, 720, "U008")], [],
        [f"data strength = scalar:FLOAT32,{tc}", "data min_distance = scalar:FLOAT32,6.0",
         "data sensitivity = scalar:FLOAT32,0.05", f"data grad_size = scalar:INT32,{gs}",
         f"data block_size = scalar:INT32,{gs}", "data num_corners = scalar:SIZE,0"],
        "node org.khronos.openvx.harris_corners input_1 strength min_distance sensitivity grad_size block_size "
        "output_1 num_corners", arrays=[("output_1", 60000)]))
for sup in (0, 1):
    CASES.append(Case(
        f"vision/FastCorners_XY_U8_{'Supression' if sup else 'NoSupression'}", [("input_1", 1280, 720, "U008")], [],
        ["data strength = scalar:FLOAT32,45.0", f"data nonmax = scalar:BOOL,{sup}", "data num_corners = scalar:SIZE,0"],
        "node org.khronos.openvx.fast_corners input_1 strength nonmax output_1 num_corners",
        arrays=[("output_1", 400000)]))


def case_ids():
    return [c.name.split("/")[1] for c in CASES]


def write_inputs(case: Case, tmp: str, seed: int = 0):
    """Seeded random frames for the case's inputs (raw, planes one after the other)."""
    rng = np.random.default_rng(seed + sum(map(ord, case.name)))
    paths = {}
    for name, w, h, fmt in case.inputs:
        p = os.path.join(tmp, f"in_{name}.raw")
        rng.integers(0, 256, frame_bytes(w, h, fmt), dtype=np.uint8).tofile(p)
        paths[name] = p
    return paths


def gdf(case: Case, tmp: str, mode: str) -> str:
    """GDF text of the case; mode 'write' saves the outputs, 'compare' checks them."""
    lines = []
    for name, w, h, fmt in case.inputs:
        lines.append(f"data {name} = image:{w},{h},{fmt}:READ,{os.path.join(tmp, 'in_' + name + '.raw')}")
    lines += case.lines
    for name, w, h, fmt, margin in case.outputs:
        ref = os.path.join(tmp, f"ref_{name}.raw")
        if mode == "write":
            io = f"WRITE,{ref}"
        else:
            io = f"COMPARE,{ref},rect{{{margin};{margin};{w - margin};{h - margin}}}"
        lines.append(f"data {name} = image:{w},{h},{fmt}:{io}")
    for name, cap in case.arrays:
        ref = os.path.join(tmp, f"ref_{name}.bin")
        lines.append(f"data {name} = array:KEYPOINT,{cap}:{'WRITE' if mode == 'write' else 'COMPARE'},{ref}")
    lines.append(case.node)
    return "\n".join(lines) + "\n"
