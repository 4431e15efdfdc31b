// Generated by gen_pow_tables.py (do not edit): the tables and constants of the Delinearize
// powf as bit patterns of doubles; see the generator for what each holds.
#pragma once

#define TW_POW_THIRD 0x3fd5555555555555ull
#define TW_POW_SIXTH 0x3fc5555555555555ull
#define TW_POW_LN2 0x3fe62e42fefa39efull
#define TW_POW_LN2_64 0x3f862e42fefa39efull
#define TW_POW_K64 0x40571547652b82feull
#define TW_POW_LIM_HI 0x40562e4300000000ull
#define TW_POW_LIM_LO 0xc059d1da00000000ull
#define TW_POW_C0 0x3f89999999bac6d4ull
#define TW_POW_C1 0x3f3c8034c85dfff0ull
#define TW_POW_A0 0x3fb55555555554e6ull
#define TW_POW_A1 0x3f62492307f1519full

#define TW_POW_RCP_INIT { \
    0x4000000000000000ull, 0x3fffe01fe01fe020ull, 0x3fffc07f01fc07f0ull, \
    0x3fffa11caa01fa12ull, 0x3fff81f81f81f820ull, 0x3fff6310aca0dbb5ull, \
    0x3fff44659e4a4271ull, 0x3fff25f644230ab5ull, 0x3fff07c1f07c1f08ull, \
    0x3ffee9c7f8458e02ull, 0x3ffecc07b301ecc0ull, 0x3ffeae807aba01ebull, \
    0x3ffe9131abf0b767ull, 0x3ffe741aa59750e4ull, 0x3ffe573ac901e574ull, \
    0x3ffe3a9179dc1a73ull, 0x3ffe1e1e1e1e1e1eull, 0x3ffe01e01e01e01eull, \
    0x3ffde5d6e3f8868aull, 0x3ffdca01dca01dcaull, 0x3ffdae6076b981dbull, \
    0x3ffd92f2231e7f8aull, 0x3ffd77b654b82c34ull, 0x3ffd5cac807572b2ull, \
    0x3ffd41d41d41d41dull, 0x3ffd272ca3fc5b1aull, 0x3ffd0cb58f6ec074ull, \
    0x3ffcf26e5c44bfc6ull, 0x3ffcd85689039b0bull, 0x3ffcbe6d9601cbe7ull, \
    0x3ffca4b3055ee191ull, 0x3ffc8b265afb8a42ull, 0x3ffc71c71c71c71cull, \
    0x3ffc5894d10d4986ull, 0x3ffc3f8f01c3f8f0ull, 0x3ffc26b5392ea01cull, \
    0x3ffc0e070381c0e0ull, 0x3ffbf583ee868d8bull, 0x3ffbdd2b899406f7ull, \
    0x3ffbc4fd65883e7bull, 0x3ffbacf914c1bad0ull, 0x3ffb951e2b18ff23ull, \
    0x3ffb7d6c3dda338bull, 0x3ffb65e2e3beee05ull, 0x3ffb4e81b4e81b4full, \
    0x3ffb37484ad806ceull, 0x3ffb2036406c80d9ull, 0x3ffb094b31d922a4ull, \
    0x3ffaf286bca1af28ull, 0x3ffadbe87f94905eull, 0x3ffac5701ac5701bull, \
    0x3ffaaf1d2f87ebfdull, 0x3ffa98ef606a63beull, 0x3ffa82e65130e159ull, \
    0x3ffa6d01a6d01a6dull, 0x3ffa574107688a4aull, 0x3ffa41a41a41a41aull, \
    0x3ffa2c2a87c51ca0ull, 0x3ffa16d3f97a4b02ull, 0x3ffa01a01a01a01aull, \
    0x3ff9ec8e951033d9ull, 0x3ff9d79f176b682dull, 0x3ff9c2d14ee4a102ull, \
    0x3ff9ae24ea5510daull, 0x3ff999999999999aull, 0x3ff9852f0d8ec0ffull, \
    0x3ff970e4f80cb872ull, 0x3ff95cbb0be377aeull, 0x3ff948b0fcd6e9e0ull, \
    0x3ff934c67f9b2ce6ull, 0x3ff920fb49d0e229ull, 0x3ff90d4f120190d5ull, \
    0x3ff8f9c18f9c18faull, 0x3ff8e6527af1373full, 0x3ff8d3018d3018d3ull, \
    0x3ff8bfce8062ff3aull, 0x3ff8acb90f6bf3aaull, 0x3ff899c0f601899cull, \
    0x3ff886e5f0abb04aull, 0x3ff87427bcc092b9ull, 0x3ff8618618618618ull, \
    0x3ff84f00c2780614ull, 0x3ff83c977ab2beddull, 0x3ff82a4a0182a4a0ull, \
    0x3ff8181818181818ull, 0x3ff8060180601806ull, 0x3ff7f405fd017f40ull, \
    0x3ff7e225515a4f1dull, 0x3ff7d05f417d05f4ull, 0x3ff7beb3922e017cull, \
    0x3ff7ad2208e0ecc3ull, 0x3ff79baa6bb6398bull, 0x3ff78a4c8178a4c8ull, \
    0x3ff77908119ac60dull, 0x3ff767dce434a9b1ull, 0x3ff756cac201756dull, \
    0x3ff745d1745d1746ull, 0x3ff734f0c541fe8dull, 0x3ff724287f46debcull, \
    0x3ff713786d9c7c09ull, 0x3ff702e05c0b8170ull, 0x3ff6f26016f26017ull, \
    0x3ff6e1f76b4337c7ull, 0x3ff6d1a62681c861ull, 0x3ff6c16c16c16c17ull, \
    0x3ff6b1490aa31a3dull, 0x3ff6a13cd1537290ull, 0x3ff691473a88d0c0ull, \
    0x3ff6816816816817ull, 0x3ff6719f3601671aull, 0x3ff661ec6a5122f9ull, \
    0x3ff6524f853b4aa3ull, 0x3ff642c8590b2164ull, 0x3ff63356b88ac0deull, \
    0x3ff623fa77016240ull, 0x3ff614b36831ae94ull, 0x3ff6058160581606ull, \
    0x3ff5f66434292dfcull, 0x3ff5e75bb8d015e7ull, 0x3ff5d867c3ece2a5ull, \
    0x3ff5c9882b931057ull, 0x3ff5babcc647fa91ull, 0x3ff5ac056b015ac0ull, \
    0x3ff59d61f123ccaaull, 0x3ff58ed2308158edull, 0x3ff5805601580560ull, \
    0x3ff571ed3c506b3aull, 0x3ff56397ba7c52e2ull, 0x3ff5555555555555ull, \
    0x3ff54725e6bb82feull, 0x3ff5390948f40febull, 0x3ff52aff56a8054bull, \
    0x3ff51d07eae2f815ull, 0x3ff50f22e111c4c5ull, 0x3ff5015015015015ull, \
    0x3ff4f38f62dd4c9bull, 0x3ff4e5e0a72f0539ull, 0x3ff4d843bedc2c4cull, \
    0x3ff4cab88725af6eull, 0x3ff4bd3edda68fe1ull, 0x3ff4afd6a052bf5bull, \
    0x3ff4a27fad76014aull, 0x3ff49539e3b2d067ull, 0x3ff4880522014880ull, \
    0x3ff47ae147ae147bull, 0x3ff46dce34596066ull, 0x3ff460cbc7f5cf9aull, \
    0x3ff453d9e2c776caull, 0x3ff446f86562d9fbull, 0x3ff43a2730abee4dull, \
    0x3ff42d6625d51f87ull, 0x3ff420b5265e5951ull, 0x3ff4141414141414ull, \
    0x3ff40782d10e6566ull, 0x3ff3fb013fb013fbull, 0x3ff3ee8f42a5af07ull, \
    0x3ff3e22cbce4a902ull, 0x3ff3d5d991aa75c6ull, 0x3ff3c995a47babe7ull, \
    0x3ff3bd60d9232955ull, 0x3ff3b13b13b13b14ull, 0x3ff3a524387ac822ull, \
    0x3ff3991c2c187f63ull, 0x3ff38d22d366088eull, 0x3ff3813813813814ull, \
    0x3ff3755bd1c945eeull, 0x3ff3698df3de0748ull, 0x3ff35dce5f9f2af8ull, \
    0x3ff3521cfb2b78c1ull, 0x3ff34679ace01346ull, 0x3ff33ae45b57bcb2ull, \
    0x3ff32f5ced6a1dfaull, 0x3ff323e34a2b10bfull, 0x3ff3187758e9ebb6ull, \
    0x3ff30d190130d190ull, 0x3ff301c82ac40260ull, 0x3ff2f684bda12f68ull, \
    0x3ff2eb4ea1fed14bull, 0x3ff2e025c04b8097ull, 0x3ff2d50a012d50a0ull, \
    0x3ff2c9fb4d812ca0ull, 0x3ff2bef98e5a3711ull, 0x3ff2b404ad012b40ull, \
    0x3ff2a91c92f3c105ull, 0x3ff29e4129e4129eull, 0x3ff293725bb804a5ull, \
    0x3ff288b01288b013ull, 0x3ff27dfa38a1ce4dull, 0x3ff27350b8812735ull, \
    0x3ff268b37cd60127ull, 0x3ff25e22708092f1ull, 0x3ff2539d7e9177b2ull, \
    0x3ff2492492492492ull, 0x3ff23eb79717605bull, 0x3ff23456789abcdfull, \
    0x3ff22a0122a0122aull, 0x3ff21fb78121fb78ull, 0x3ff21579804855e6ull, \
    0x3ff20b470c67c0d9ull, 0x3ff2012012012012ull, 0x3ff1f7047dc11f70ull, \
    0x3ff1ecf43c7fb84cull, 0x3ff1e2ef3b3fb874ull, 0x3ff1d8f5672e4abdull, \
    0x3ff1cf06ada2811dull, 0x3ff1c522fc1ce059ull, 0x3ff1bb4a4046ed29ull, \
    0x3ff1b17c67f2bae3ull, 0x3ff1a7b9611a7b96ull, 0x3ff19e0119e0119eull, \
    0x3ff19453808ca29cull, 0x3ff18ab083902bdbull, 0x3ff1811811811812ull, \
    0x3ff1778a191bd684ull, 0x3ff16e0689427379ull, 0x3ff1648d50fc3201ull, \
    0x3ff15b1e5f75270dull, 0x3ff151b9a3fdd5c9ull, 0x3ff1485f0e0acd3bull, \
    0x3ff13f0e8d344724ull, 0x3ff135c81135c811ull, 0x3ff12c8b89edc0acull, \
    0x3ff12358e75d3033ull, 0x3ff11a3019a74826ull, 0x3ff1111111111111ull, \
    0x3ff107fbbe011080ull, 0x3ff0fef010fef011ull, 0x3ff0f5edfab325a2ull, \
    0x3ff0ecf56be69c90ull, 0x3ff0e40655826011ull, 0x3ff0db20a88f4696ull, \
    0x3ff0d24456359e3aull, 0x3ff0c9714fbcda3bull, 0x3ff0c0a7868b4171ull, \
    0x3ff0b7e6ec259dc8ull, 0x3ff0af2f722eecb5ull, 0x3ff0a6810a6810a7ull, \
    0x3ff09ddba6af8360ull, 0x3ff0953f39010954ull, 0x3ff08cabb37565e2ull, \
    0x3ff0842108421084ull, 0x3ff07b9f29b8eae2ull, 0x3ff073260a47f7c6ull, \
    0x3ff06ab59c7912fbull, 0x3ff0624dd2f1a9fcull, 0x3ff059eea0727586ull, \
    0x3ff05197f7d73404ull, 0x3ff04949cc1664c5ull, 0x3ff0410410410410ull, \
    0x3ff038c6b78247fcull, 0x3ff03091b51f5e1aull, 0x3ff02864fc7729e9ull, \
    0x3ff0204081020408ull, 0x3ff0182436517a37ull, 0x3ff0101010101010ull, \
    0x3ff0080402010080ull, 0x3ff0000000000000ull \
}

#define TW_POW_LOG_INIT { \
    0x0000000000000000ull, 0x3f6ff00aa2b10bc0ull, 0x3f7fe02a6b106789ull, \
    0x3f87dc475f810a77ull, 0x3f8fc0a8b0fc03e4ull, 0x3f93cea44346a575ull, \
    0x3f97b91b07d5b11bull, 0x3f9b9fc027af9198ull, 0x3f9f829b0e783300ull, \
    0x3fa1b0d98923d980ull, 0x3fa39e87b9febd60ull, 0x3fa58a5bafc8e4d5ull, \
    0x3fa77458f632dcfcull, 0x3fa95c830ec8e3ebull, 0x3fab42dd711971bfull, \
    0x3fad276b8adb0b52ull, 0x3faf0a30c01162a6ull, 0x3fb075983598e471ull, \
    0x3fb16536eea37ae1ull, 0x3fb253f62f0a1417ull, 0x3fb341d7961bd1d1ull, \
    0x3fb42edcbea646f0ull, 0x3fb51b073f06183full, 0x3fb60658a93750c4ull, \
    0x3fb6f0d28ae56b4cull, 0x3fb7da766d7b12cdull, 0x3fb8c345d6319b21ull, \
    0x3fb9ab42462033adull, 0x3fba926d3a4ad563ull, 0x3fbb78c82bb0eda1ull, \
    0x3fbc5e548f5bc743ull, 0x3fbd4313d66cb35dull, 0x3fbe27076e2af2e6ull, \
    0x3fbf0a30c01162a6ull, 0x3fbfec9131dbeabbull, 0x3fc0671512ca596eull, \
    0x3fc0d77e7cd08e59ull, 0x3fc14785846742acull, 0x3fc1b72ad52f67a0ull, \
    0x3fc2266f190a5acbull, 0x3fc29552f81ff523ull, 0x3fc303d718e47fd3ull, \
    0x3fc371fc201e8f74ull, 0x3fc3dfc2b0ecc62aull, 0x3fc44d2b6ccb7d1eull, \
    0x3fc4ba36f39a55e5ull, 0x3fc526e5e3a1b438ull, 0x3fc59338d9982086ull, \
    0x3fc5ff3070a793d4ull, 0x3fc66acd4272ad51ull, 0x3fc6d60fe719d21dull, \
    0x3fc740f8f54037a5ull, 0x3fc7ab890210d909ull, 0x3fc815c0a14357ebull, \
    0x3fc87fa06520c911ull, 0x3fc8e928de886d41ull, 0x3fc9525a9cf456b4ull, \
    0x3fc9bb362e7dfb83ull, 0x3fca23bc1fe2b563ull, 0x3fca8becfc882f19ull, \
    0x3fcaf3c94e80bff3ull, 0x3fcb5b519e8fb5a4ull, 0x3fcbc286742d8cd6ull, \
    0x3fcc2968558c18c1ull, 0x3fcc8ff7c79a9a22ull, 0x3fccf6354e09c5dcull, \
    0x3fcd5c216b4fbb91ull, 0x3fcdc1bca0abec7dull, 0x3fce27076e2af2e6ull, \
    0x3fce8c0252aa5a60ull, 0x3fcef0adcbdc5936ull, 0x3fcf550a564b7b37ull, \
    0x3fcfb9186d5e3e2bull, 0x3fd00e6c45ad501dull, 0x3fd0402594b4d041ull, \
    0x3fd071b85fcd590dull, 0x3fd0a324e27390e3ull, 0x3fd0d46b579ab74bull, \
    0x3fd1058bf9ae4ad5ull, 0x3fd136870293a8b0ull, 0x3fd1675cababa60eull, \
    0x3fd1980d2dd4236full, 0x3fd1c898c16999fbull, 0x3fd1f8ff9e48a2f3ull, \
    0x3fd22941fbcf7966ull, 0x3fd2596010df763aull, 0x3fd2895a13de86a3ull, \
    0x3fd2b9303ab89d25ull, 0x3fd2e8e2bae11d31ull, 0x3fd31871c9544185ull, \
    0x3fd347dd9a987d55ull, 0x3fd3772662bfd85bull, 0x3fd3a64c556945eaull, \
    0x3fd3d54fa5c1f710ull, 0x3fd404308686a7e4ull, 0x3fd432ef2a04e814ull, \
    0x3fd4618bc21c5ec2ull, 0x3fd49006804009d1ull, 0x3fd4be5f957778a1ull, \
    0x3fd4ec973260026aull, 0x3fd51aad872df82dull, 0x3fd548a2c3add263ull, \
    0x3fd5767717455a6cull, 0x3fd5a42ab0f4cfe2ull, 0x3fd5d1bdbf5809caull, \
    0x3fd5ff3070a793d4ull, 0x3fd62c82f2b9c795ull, 0x3fd659b57303e1f3ull, \
    0x3fd686c81e9b14afull, 0x3fd6b3bb2235943eull, 0x3fd6e08eaa2ba1e4ull, \
    0x3fd70d42e2789236ull, 0x3fd739d7f6bbd007ull, 0x3fd7664e1239dbcfull, \
    0x3fd792a55fdd47a2ull, 0x3fd7bede0a37afc0ull, 0x3fd7eaf83b82afc3ull, \
    0x3fd816f41da0d496ull, 0x3fd842d1da1e8b17ull, 0x3fd86e919a330ba0ull, \
    0x3fd89a3386c1425bull, 0x3fd8c5b7c858b48bull, 0x3fd8f11e873662c7ull, \
    0x3fd91c67eb45a83eull, 0x3fd947941c2116fbull, 0x3fd972a341135158ull, \
    0x3fd99d958117e08bull, 0x3fd9c86b02dc0863ull, 0x3fd9f323ecbf984cull, \
    0x3fda1dc064d5b995ull, 0x3fda484090e5bb0aull, 0x3fda72a4966bd9eaull, \
    0x3fda9cec9a9a084aull, 0x3fdac718c258b0e4ull, 0x3fdaf1293247786bull, \
    0x3fdb1b1e0ebdfc5bull, 0x3fdb44f77bcc8f63ull, 0x3fdb6eb59d3cf35eull, \
    0x3fdb9858969310fbull, 0x3fdbc1e08b0dad0aull, 0x3fdbeb4d9da71b7cull, \
    0x3fdc149ff115f027ull, 0x3fdc3dd7a7cdad4dull, 0x3fdc66f4e3ff6ff8ull, \
    0x3fdc8ff7c79a9a22ull, 0x3fdcb8e0744d7acaull, 0x3fdce1af0b85f3ebull, \
    0x3fdd0a63ae721e64ull, 0x3fdd32fe7e00ebd5ull, 0x3fdd5b7f9ae2c684ull, \
    0x3fdd83e7258a2f3eull, 0x3fddac353e2c5954ull, 0x3fddd46a04c1c4a1ull, \
    0x3fddfc859906d5b5ull, 0x3fde24881a7c6c26ull, 0x3fde4c71a8687704ull, \
    0x3fde744261d68788ull, 0x3fde9bfa659861f5ull, 0x3fdec399d2468cc0ull, \
    0x3fdeeb20c640ddf4ull, 0x3fdf128f5faf06edull, 0x3fdf39e5bc811e5cull, \
    0x3fdf6123fa7028acull, 0x3fdf884a36fe9ec2ull, 0x3fdfaf588f78f31full, \
    0x3fdfd64f20f61572ull, 0x3fdffd2e0857f498ull, 0x3fe011fab125ff8aull, \
    0x3fe02552a5a5d0ffull, 0x3fe0389eefce633bull, 0x3fe04bdf9da926d2ull, \
    0x3fe05f14bd26459cull, 0x3fe0723e5c1cdf40ull, 0x3fe0855c884b450eull, \
    0x3fe0986f4f573521ull, 0x3fe0ab76bece14d2ull, 0x3fe0be72e4252a83ull, \
    0x3fe0d163ccb9d6b8ull, 0x3fe0e44985d1cc8cull, 0x3fe0f7241c9b497dull, \
    0x3fe109f39e2d4c97ull, 0x3fe11cb81787ccf8ull, 0x3fe12f719593efbcull, \
    0x3fe1422025243d45ull, 0x3fe154c3d2f4d5eaull, 0x3fe1675cababa60eull, \
    0x3fe179eabbd899a1ull, 0x3fe18c6e0ff5cf06ull, 0x3fe19ee6b467c96full, \
    0x3fe1b154b57da29full, 0x3fe1c3b81f713c25ull, 0x3fe1d610fe677003ull, \
    0x3fe1e85f5e7040d0ull, 0x3fe1faa34b87094cull, 0x3fe20cdcd192ab6eull, \
    0x3fe21f0bfc65beecull, 0x3fe23130d7bebf43ull, 0x3fe2434b6f483934ull, \
    0x3fe2555bce98f7cbull, 0x3fe26762013430e0ull, 0x3fe2795e1289b11bull, \
    0x3fe28b500df60783ull, 0x3fe29d37fec2b08bull, 0x3fe2af15f02640adull, \
    0x3fe2c0e9ed448e8cull, 0x3fe2d2b4012edc9eull, 0x3fe2e47436e40268ull, \
    0x3fe2f62a99509546ull, 0x3fe307d7334f10beull, 0x3fe3197a0fa7fe6aull, \
    0x3fe32b1339121d71ull, 0x3fe33ca2ba328995ull, 0x3fe34e289d9ce1d3ull, \
    0x3fe35fa4edd36ea0ull, 0x3fe37117b54747b6ull, 0x3fe38280fe58797full, \
    0x3fe393e0d3562a1aull, 0x3fe3a5373e7ebdfaull, 0x3fe3b68449fffc23ull, \
    0x3fe3c7c7fff73206ull, 0x3fe3d9026a7156fbull, 0x3fe3ea33936b2f5cull, \
    0x3fe3fb5b84d16f42ull, 0x3fe40c7a4880dce9ull, 0x3fe41d8fe84672aeull, \
    0x3fe42e9c6ddf80bfull, 0x3fe43f9fe2f9ce67ull, 0x3fe4509a5133bb0aull, \
    0x3fe4618bc21c5ec2ull, 0x3fe472743f33aaadull, 0x3fe48353d1ea88dfull, \
    0x3fe4942a83a2fc07ull, 0x3fe4a4f85db03ebbull, 0x3fe4b5bd6956e274ull, \
    0x3fe4c679afccee3aull, 0x3fe4d72d3a39fd00ull, 0x3fe4e7d811b75bb1ull, \
    0x3fe4f87a3f5026e9ull, 0x3fe50913cc01686bull, 0x3fe519a4c0ba3446ull, \
    0x3fe52a2d265bc5abull, 0x3fe53aad05b99b7dull, 0x3fe54b2467999498ull, \
    0x3fe55b9354b40bcdull, 0x3fe56bf9d5b3f399ull, 0x3fe57c57f336f191ull, \
    0x3fe58cadb5cd7989ull, 0x3fe59cfb25fae87eull, 0x3fe5ad404c359f2dull, \
    0x3fe5bd7d30e71c73ull, 0x3fe5cdb1dc6c1765ull, 0x3fe5ddde57149923ull, \
    0x3fe5ee02a9241675ull, 0x3fe5fe1edad18919ull, 0x3fe60e32f44788d9ull, \
    0x3fe61e3efda46467ull, 0x3fe62e42fefa39efull \
}

#define TW_POW_EXP2_INIT { \
    0x3ff0000000000000ull, 0x3ff02c9a3e778061ull, 0x3ff059b0d3158574ull, \
    0x3ff0874518759bc8ull, 0x3ff0b5586cf9890full, 0x3ff0e3ec32d3d1a2ull, \
    0x3ff11301d0125b51ull, 0x3ff1429aaea92de0ull, 0x3ff172b83c7d517bull, \
    0x3ff1a35beb6fcb75ull, 0x3ff1d4873168b9aaull, 0x3ff2063b88628cd6ull, \
    0x3ff2387a6e756238ull, 0x3ff26b4565e27cddull, 0x3ff29e9df51fdee1ull, \
    0x3ff2d285a6e4030bull, 0x3ff306fe0a31b715ull, 0x3ff33c08b26416ffull, \
    0x3ff371a7373aa9cbull, 0x3ff3a7db34e59ff7ull, 0x3ff3dea64c123422ull, \
    0x3ff4160a21f72e2aull, 0x3ff44e086061892dull, 0x3ff486a2b5c13cd0ull, \
    0x3ff4bfdad5362a27ull, 0x3ff4f9b2769d2ca7ull, 0x3ff5342b569d4f82ull, \
    0x3ff56f4736b527daull, 0x3ff5ab07dd485429ull, 0x3ff5e76f15ad2148ull, \
    0x3ff6247eb03a5585ull, 0x3ff6623882552225ull, 0x3ff6a09e667f3bcdull, \
    0x3ff6dfb23c651a2full, 0x3ff71f75e8ec5f74ull, 0x3ff75feb564267c9ull, \
    0x3ff7a11473eb0187ull, 0x3ff7e2f336cf4e62ull, 0x3ff82589994cce13ull, \
    0x3ff868d99b4492edull, 0x3ff8ace5422aa0dbull, 0x3ff8f1ae99157736ull, \
    0x3ff93737b0cdc5e5ull, 0x3ff97d829fde4e50ull, 0x3ff9c49182a3f090ull, \
    0x3ffa0c667b5de565ull, 0x3ffa5503b23e255dull, 0x3ffa9e6b5579fdbfull, \
    0x3ffae89f995ad3adull, 0x3ffb33a2b84f15fbull, 0x3ffb7f76f2fb5e47ull, \
    0x3ffbcc1e904bc1d2ull, 0x3ffc199bdd85529cull, 0x3ffc67f12e57d14bull, \
    0x3ffcb720dcef9069ull, 0x3ffd072d4a07897cull, 0x3ffd5818dcfba487ull, \
    0x3ffda9e603db3285ull, 0x3ffdfc97337b9b5full, 0x3ffe502ee78b3ff6ull, \
    0x3ffea4afa2a490daull, 0x3ffefa1bee615a27ull, 0x3fff50765b6e4540ull, \
    0x3fffa7c1819e90d8ull \
}
