// The glibc logf exception table (gen_logf_table.c output, pairs of uint32 input bits and glibc
// result bits), embedded in the library; the build assembles this with the table's directory on
// the assembler's include path.
    .section .rodata
    .balign 16
    .globl tw_logf_table
    .hidden tw_logf_table
tw_logf_table:
    .incbin "logf_table.bin"
    .globl tw_logf_table_end
    .hidden tw_logf_table_end
tw_logf_table_end:
    .section .note.GNU-stack,"",@progbits
