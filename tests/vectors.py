"""Hand-built known-answer streams, one per header type and per kept reference quirk.

Each entry: (codec, elem_bytes, stream bytes, expected values).  The expected values are
worked out by hand from the stream grammar (comments show the arithmetic), independently
of both decoders, and both the CPU oracle and the GPU kernels must reproduce them.
"""
RLEV1, RLEV2 = 0, 1

VECTORS = {
    # --- ORC RLE v1 (include/rlev1/decoder.h:588-798) ---------------------------------------
    # 0xFE = -2: two literal varints 5 and 0x80 0x01 = 128; 0x00: run of 3 with delta 0xFF = -1
    # from base 10.
    "v1_literals_and_run": (RLEV1, 8, [0xFE, 0x05, 0x80, 0x01, 0x00, 0xFF, 0x0A], [5, 128, 10, 9, 8]),
    # run header 126 = 129 values, delta +2 from base 0x81 0x01 = 129
    "v1_long_run": (RLEV1, 8, [126, 0x02, 0x81, 0x01], [129 + 2 * i for i in range(129)]),
    # 16-bit elements: literal 0xFF 0xFF 0x03 = 65535; run of 3 from 65535 with delta +1 wraps
    "v1_u16_wrap": (RLEV1, 2, [0xFF, 0xFF, 0xFF, 0x03, 0x00, 0x01, 0xFF, 0xFF, 0x03], [65535, 65535, 0, 1]),
    # a 10-byte varint holding 2^63 + 1 in 64-bit elements
    "v1_max_varint": (RLEV1, 8, [0xFF, 0x81] + [0x80] * 8 + [0x01], [(1 << 63) + 1]),

    # --- ORC RLE v2 (include/rlev2/decoder_new.h:909-1187) ----------------------------------
    # SHORT_REPEAT 0x0A: width (1+1) bytes, count 2+3 = 5, value 0x2710 = 10000
    "v2_short_repeat": (RLEV2, 8, [0x0A, 0x27, 0x10], [10000] * 5),
    # DIRECT 0x5E 0x03: width code 15 = 16 bits, 4 values big-endian
    "v2_direct16": (RLEV2, 8, [0x5E, 0x03, 0x00, 0x17, 0x00, 0x2A, 0x01, 0x00, 0xFF, 0xFF], [23, 42, 256, 65535]),
    # DIRECT width code 2 = 3 bits, 5 values 7,0,5,1,6 packed MSB first: 111 000 101 001 110 -> 0xE2 0x9C
    "v2_direct3": (RLEV2, 4, [0x44, 0x04, 0xE2, 0x9C], [7, 0, 5, 1, 6]),
    # DELTA fixed step: width code 0, 5 values, base 2, base delta zigzag(2) = 4
    "v2_delta_fixed": (RLEV2, 8, [0xC0, 0x04, 0x02, 0x04], [2, 4, 6, 8, 10]),
    # DELTA packed: width code 3 = 4 bits, 5 values, base 1, delta zigzag(1)=2, deltas 2,0,5
    "v2_delta_packed": (RLEV2, 8, [0xC6, 0x04, 0x01, 0x02, 0x20, 0x50], [1, 2, 4, 4, 9]),
    # DELTA decreasing, width code 31 = 64 bits, 4 values: base 100, base delta zigzag 5 = -3;
    # the unsigned base delta is non-zero so the multiplier is +1 and the packed deltas are
    # stored as 2^64-3 and 2^64-4 (modular additions of -3 and -4).
    "v2_delta_down64": (RLEV2, 8, [0xFE, 0x03, 0x64, 0x05]
                        + [0xFF] * 7 + [0xFD] + [0xFF] * 7 + [0xFC], [100, 97, 94, 90]),
    # PATCHED_BASE: fbw 8 (code 7), 4 values, base width 1 byte, patch width 4 (code 3),
    # gap width 2, one patch; base 10; values 1,2,3,4; patch entry (6 bits) = gap 2 << 4 | 5
    # -> value 2 becomes ((13 - 10) | 5 << 8) + 10 = 1293
    "v2_patched": (RLEV2, 8, [0x8E, 0x03, 0x03, 0x21, 0x0A, 0x01, 0x02, 0x03, 0x04, 0x94], [11, 12, 1293, 14]),
    # quirk: a DIRECT length field of 255 decodes to 0 values in a uint8_t; then SHORT_REPEAT of 7
    "v2_quirk_len_wrap": (RLEV2, 8, [0x41, 0xFF, 0x00, 0x07], [7, 7, 7]),
    # quirk: DELTA with length field 0 (one value): "len -= 2" wraps to 255 more values
    "v2_quirk_delta_wrap": (RLEV2, 8, [0xC0, 0x00, 0x05, 0x02], [5 + i for i in range(257)]),
    # quirk: patch width 40 (code 28) is masked to 32 bits; entry 48 bits = gap 1 << 40 |
    # 0x1_0000_0001 -> the patch becomes 1 and value 1 becomes 2 | 1 << 8 = 258
    "v2_quirk_patch_mask": (RLEV2, 8, [0x8E, 0x01, 0x1C, 0x01, 0x00, 0x01, 0x02,
                                       0x01, 0x01, 0x00, 0x00, 0x00, 0x01], [1, 258]),
}
